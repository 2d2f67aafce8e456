// Mixed-precision block-tridiagonal solve: the diagonal blocks are factored
// and inverted in FP32 (same kernel as the FP64 path, element type float),
// and the solution is recovered in FP64 by iterative refinement on the full
// block-tridiagonal system
//     r = b - M x          (FP64, from the FP64 blocks and off-diagonals)
//     x = x + M~^{-1} r     (block-Thomas sweeps with the FP32 inverses)
// until max|correction| <= tol * max|x|. Atmospheres whose refinement stalls
// are refactored and solved in FP64 and flagged VB_STATUS_REFINE_STALL.
// M is the system of reference solver.py:33-112: diagonal blocks A_j,
// sub-diagonal diag(sub_d[j-1]) at (j, j-1), super-diagonal diag(sup_d[j])
// at (j, j+1).
#include <cuda_runtime.h>

#include "vb_common.cuh"
#include "vb_launch.cuh"

namespace vb {

constexpr int REFINE_THREADS = 256;
constexpr int REFINE_WARPS = REFINE_THREADS / 32;

// y[i] = sum_m A[i][m] v[m] for an n x n block of row stride ld (one warp per
// row, lanes over columns); v and y in shared memory.
template <typename T>
__device__ inline void block_mv(const T* __restrict__ A, int n, int ld, const double* v, double* y) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = warp; i < n; i += REFINE_WARPS) {
    double s = 0.0;
    for (int m = lane; m < n; m += 32) s = fma((double)A[(int64_t)i * ld + m], v[m], s);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) y[i] = s;
  }
}

// One pass of refinement for every atmosphere (CTA per atmosphere). first:
// x is taken as 0 (the pass is the plain solve). state[b]: 1 once converged
// (later passes skip it). only != nullptr: atmospheres with only[b] == 0 skip.
template <typename R>
__global__ void __launch_bounds__(REFINE_THREADS)
refine_kernel(Batch B, double* __restrict__ ws, const R* __restrict__ inv, const double* __restrict__ rhs,
              double* __restrict__ x, int32_t* __restrict__ state, int32_t* __restrict__ passes, double tol,
              int first, const int32_t* __restrict__ only) {
  __shared__ double sx[VB_MAX_NI], sv[VB_MAX_NI], sr[VB_MAX_NI], su[VB_MAX_NI];
  __shared__ double red[REFINE_WARPS][2];
  const int b = blockIdx.x;
  if (only && only[b] == 0) return;
  if (!first && state[b] == 1) return;
  const Geo g = geo_of(B, b);
  const int n = B.ni, nz = g.nz, ld = B.ld;
  WsView w = ws_view(ws, g, n, ld);
  const R* Ib = inv + g.z0 * n * ld;
  const double* bb = rhs + g.z0 * n;
  double* xb = x + g.z0 * n;
  double* rp = w.rmod;   // forward-eliminated residual, [nz][ni]
  // ---- forward: r_j = b_j - (M x)_j, r'_j = r_j - sub[j-1] o (Inv_{j-1} r'_{j-1})
  for (int j = 0; j < nz; ++j) {
    if (!first)
      for (int i = threadIdx.x; i < n; i += blockDim.x) sx[i] = xb[(int64_t)j * n + i];
    __syncthreads();
    if (!first) block_mv(w.inv + (int64_t)j * n * ld, n, ld, sx, su);   // A_j x_j (FP64 blocks)
    if (j > 0) block_mv(Ib + (int64_t)(j - 1) * n * ld, n, ld, sr, sv);  // Inv_{j-1} r'_{j-1}
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double r = bb[(int64_t)j * n + i];
      if (!first) {
        double mx = su[i];
        if (j > 0) mx = mx + w.subn[(int64_t)(j - 1) * n + i] * xb[(int64_t)(j - 1) * n + i];
        if (j < nz - 1) mx = mx + w.supn[(int64_t)j * n + i] * xb[(int64_t)(j + 1) * n + i];
        r = r - mx;
      }
      if (j > 0) r = r - w.subn[(int64_t)(j - 1) * n + i] * sv[i];
      rp[(int64_t)j * n + i] = r;
      sr[i] = r;
    }
    __syncthreads();
  }
  // ---- backward: c_j = Inv_j (r'_j - sup[j] o c_{j+1}); x_j += c_j
  double cmax = 0.0, xmax = 0.0;
  for (int j = nz - 1; j >= 0; --j) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double v = rp[(int64_t)j * n + i];
      if (j < nz - 1) v = v - w.supn[(int64_t)j * n + i] * su[i];
      sv[i] = v;
    }
    __syncthreads();
    block_mv(Ib + (int64_t)j * n * ld, n, ld, sv, sr);   // c_j
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double c = sr[i];
      const double xn = (first ? 0.0 : xb[(int64_t)j * n + i]) + c;
      xb[(int64_t)j * n + i] = xn;
      su[i] = c;
      cmax = fmax(cmax, fabs(c));
      xmax = fmax(xmax, fabs(xn));
      if (!isfinite(xn)) cmax = INFINITY;
    }
    __syncthreads();
  }
  // ---- convergence of this atmosphere
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, off));
    xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, off));
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5][0] = cmax;
    red[threadIdx.x >> 5][1] = xmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double cm = red[0][0], xm = red[0][1];
    for (int q = 1; q < REFINE_WARPS; ++q) {
      cm = fmax(cm, red[q][0]);
      xm = fmax(xm, red[q][1]);
    }
    passes[b] += 1;
    // the first pass is the plain solve; its correction is x itself
    state[b] = (!first && cm <= tol * xm) ? 1 : 0;
  }
}

// After the FP32 passes: atmospheres that did not converge get the FP64
// fallback (fallback[b] = 1) and VB_STATUS_REFINE_STALL.
__global__ void refine_finalize_kernel(int batch, const int32_t* __restrict__ state, int32_t* __restrict__ fallback,
                                       int32_t* __restrict__ status) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const int f = state[b] == 1 ? 0 : 1;
  fallback[b] = f;
  if (f) status[b] |= VB_STATUS_REFINE_STALL;
}

template <typename R>
cudaError_t launch_refine(const Batch& B, double* ws, const R* inv, const double* rhs, double* x, int32_t* state,
                          int32_t* passes, double tol, int first, const int32_t* only, cudaStream_t st) {
  refine_kernel<R><<<B.count, REFINE_THREADS, 0, st>>>(B, ws, inv, rhs, x, state, passes, tol, first, only);
  return cudaGetLastError();
}
template cudaError_t launch_refine<float>(const Batch&, double*, const float*, const double*, double*, int32_t*,
                                          int32_t*, double, int, const int32_t*, cudaStream_t);
template cudaError_t launch_refine<double>(const Batch&, double*, const double*, const double*, double*, int32_t*,
                                           int32_t*, double, int, const int32_t*, cudaStream_t);

cudaError_t launch_refine_finalize(int batch, const int32_t* state, int32_t* fallback, int32_t* status,
                                   cudaStream_t st) {
  refine_finalize_kernel<<<(batch + 127) / 128, 128, 0, st>>>(batch, state, fallback, status);
  return cudaGetLastError();
}

}  // namespace vb
