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

// y[i] = sum_m A[i][m] (sc[m] v[m]) for an n x n block of row stride ld (one
// warp per row, lanes over columns; sc = nullptr: no column scales); v and y
// in shared memory.
template <typename T>
__device__ inline void block_mv(const T* __restrict__ A, int n, int ld, const double* v, double* y,
                                const double* __restrict__ sc = nullptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = warp; i < n; i += REFINE_WARPS) {
    double s = 0.0;
    for (int m = lane; m < n; m += 32) s = fma((double)A[(int64_t)i * ld + m], sc ? sc[m] * v[m] : v[m], s);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) y[i] = s;
  }
}

// One pass of refinement for every atmosphere (CTA per atmosphere). first:
// x is taken as 0 (the pass is the plain solve). state[b]: 1 once converged
// (later passes skip it). only != nullptr: atmospheres with only[b] == 0 skip.
// The inverses: inv (stride ld), or with mxr != nullptr (R = float) the
// row-equilibrated factors of the mixed region, A'_j^{-1} = X_j diag(r_j).
template <typename R>
__global__ void __launch_bounds__(REFINE_THREADS)
refine_kernel(Batch B, double* __restrict__ ws, const R* __restrict__ inv, const void* __restrict__ mxr,
              const double* __restrict__ rhs, double* __restrict__ x, int32_t* __restrict__ state,
              int32_t* __restrict__ passes, double tol, int first, const int32_t* __restrict__ only) {
  __shared__ double sx[VB_MAX_NI], sv[VB_MAX_NI], sr[VB_MAX_NI], su[VB_MAX_NI];
  __shared__ double red[REFINE_WARPS][2];
  const int b = blockIdx.x;
  if (only && only[b] == 0) return;
  if (!first && state[b] == 1) return;
  const Geo g = geo_of(B, b);
  const int n = B.ni, nz = g.nz, ld = B.ld;
  WsView w = ws_view(ws, g, n, ld);
  const R* Ib = inv + g.z0 * n * ld;
  int li = ld;                    // row stride of the inverses
  const double* rsc = nullptr;    // their column scales [nz][ni], if equilibrated
  if (mxr) {
    const MxView m = mx_view(const_cast<void*>(mxr), g.z0, nz, n);
    Ib = reinterpret_cast<const R*>(m.X);
    rsc = m.rs;
    li = round4(n);
  }
  const double* bb = rhs + g.z0 * n;
  double* xb = x + g.z0 * n;
  double* rp = w.rmod;   // forward-eliminated residual, [nz][ni]
  // ---- forward: r_j = b_j - (M x)_j, r'_j = r_j - sub[j-1] o (Inv_{j-1} r'_{j-1})
  for (int j = 0; j < nz; ++j) {
    if (!first)
      for (int i = threadIdx.x; i < n; i += blockDim.x) sx[i] = xb[(int64_t)j * n + i];
    __syncthreads();
    if (!first) block_mv(w.inv + (int64_t)j * n * ld, n, ld, sx, su);   // A_j x_j (FP64 blocks)
    if (j > 0)                                                           // Inv_{j-1} r'_{j-1}
      block_mv(Ib + (int64_t)(j - 1) * n * li, n, li, sr, sv, rsc ? rsc + (int64_t)(j - 1) * n : nullptr);
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
    block_mv(Ib + (int64_t)j * n * li, n, li, sv, sr, rsc ? rsc + (int64_t)j * n : nullptr);   // c_j
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
cudaError_t launch_refine(const Batch& B, double* ws, const R* inv, const void* mxr, const double* rhs, double* x,
                          int32_t* state, int32_t* passes, double tol, int first, const int32_t* only,
                          cudaStream_t st) {
  refine_kernel<R><<<B.count, REFINE_THREADS, 0, st>>>(B, ws, inv, mxr, rhs, x, state, passes, tol, first, only);
  return cudaGetLastError();
}
template cudaError_t launch_refine<float>(const Batch&, double*, const float*, const void*, const double*, double*,
                                          int32_t*, int32_t*, double, int, const int32_t*, cudaStream_t);
template cudaError_t launch_refine<double>(const Batch&, double*, const double*, const void*, const double*, double*,
                                           int32_t*, int32_t*, double, int, const int32_t*, cudaStream_t);

cudaError_t launch_refine_finalize(int batch, const int32_t* state, int32_t* fallback, int32_t* status,
                                   cudaStream_t st) {
  refine_finalize_kernel<<<(batch + 127) / 128, 128, 0, st>>>(batch, state, fallback, status);
  return cudaGetLastError();
}

// ================================================================ mixed-precision Ros2 step
// Modes of an atmosphere (mode[b]) during the solves of one step:
//   MX_REFINE  FP32 inverses, refinement still running for this right-hand side
//   MX_DONE    FP32 inverses, refinement converged for this right-hand side
//   MX_FP64    FP64 inverses in place of its blocks (the FP32 factor failed or
//              refinement stalled): solved directly, no refinement
enum MxMode { MX_REFINE = 0, MX_DONE = 1, MX_FP64 = 3 };
constexpr int MX_THREADS = 256;

__host__ __device__ inline size_t mx_al(size_t x) { return (x + 127) & ~(size_t)127; }
// Bytes of one ring stage: the FP64 block D_j (refinement passes) and one
// inverse (FP32 X_j, or the FP64 inverse of an atmosphere in MX_FP64).
__host__ __device__ inline size_t mx_stage_bytes(int ni, bool refine) {
  const size_t d = (size_t)ni * round_even(ni) * 8, x = (size_t)ni * round4(ni) * 4;
  return refine ? mx_al(d) + mx_al(x) : mx_al(d > x ? d : x);
}
__host__ __device__ inline size_t mx_pass_smem(int ni, bool refine) {
  return 2 * mx_stage_bytes(ni, refine) + 64 + 5 * VB_MAX_NI * sizeof(double);
}

// out = A v for one n x n block in shared memory (FP32 or FP64 entries, FP64
// products), four lanes per row, eight rows per warp per pass (warp-uniform passes).
template <typename T>
__device__ inline void mx_matvec(const T* __restrict__ A, int n, int lda, const double* v, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int sub = lane & 3;
  for (int i0 = warp * 8; i0 < n; i0 += nw * 8) {
    const int i = i0 + (lane >> 2);
    double s0 = 0.0, s1 = 0.0;
    if (i < n) {
      const T* row = A + i * lda;
      int m = sub;
      for (; m + 4 < n; m += 8) {
        s0 = fma((double)row[m], v[m], s0);
        s1 = fma((double)row[m + 4], v[m + 4], s1);
      }
      if (m < n) s0 = fma((double)row[m], v[m], s0);
    }
    double s = s0 + s1;
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (sub == 0 && i < n) out[i] = s;
  }
}

// One pass of the mixed-precision block solve of every atmosphere (CTA each),
// right-hand side b = the workspace's rmod rows, solution x = its k1 rows
// (xsel 0) or aux rows (xsel 1).
//  FIRST: x = M~^{-1} b with the factor's inverses (FP32 X_j with row scales,
//         or FP64 for MX_FP64 atmospheres); MX_DONE atmospheres restart as
//         MX_REFINE (a new right-hand side).
//  else:  MX_REFINE atmospheres: r = b - M x with the FP64 blocks D_j and
//         off-diagonals (the system of reference solver.py:33-112),
//         x += M~^{-1} r; MX_DONE once max|correction| <= tol max|x|.
// only != nullptr: atmospheres with only[b] == 0 skip. The blocks stream
// through a two-stage shared-memory ring filled by bulk copies with bounded
// waits (a wait that gives up drains its copies, sets VB_STATUS_WATCHDOG
// and the CTA returns). Stage s uses barrier s % 2 in phase (s / 2) % 2;
// the backward stream's stages continue the forward stream's numbering.
template <bool FIRST>
__global__ void __launch_bounds__(MX_THREADS)
mx_pass_kernel(Batch B, double* __restrict__ ws, void* __restrict__ mxr, int xsel, int32_t* __restrict__ mode,
               const int32_t* __restrict__ only, int32_t* __restrict__ passes, double tol,
               int32_t* __restrict__ status, long long wlim) {
  extern __shared__ __align__(128) char smem_raw[];
  __shared__ double red[MX_THREADS / 32][2];
  __shared__ int redb[MX_THREADS / 32];
  const int b = blockIdx.x;
  if (only && only[b] == 0) return;
  const int md = mode[b];
  if (!FIRST && md != MX_REFINE) return;
  const bool f64 = md == MX_FP64;
  const Geo g = geo_of(B, b);
  const int n = B.ni, nz = g.nz, ld = B.ld, ldf = round4(n);
  WsView w = ws_view(ws, g, n, ld);
  MxView mv = mx_view(mxr, g.z0, nz, n);
  const double* bb = w.rmod;
  double* xb = xsel ? w.aux : w.k1;
  const uint32_t dbytes = (uint32_t)(n * ld * 8);
  const uint32_t xbytes = f64 ? dbytes : (uint32_t)(n * ldf * 4);
  const size_t sb = mx_stage_bytes(n, !FIRST);
  const size_t doff = 0, xoff = FIRST ? 0 : mx_al((size_t)dbytes);   // parts of a stage
  char* ring = smem_raw;
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + 2 * sb);
  double* va = reinterpret_cast<double*>(bars + 8);   // running vector (r'_{j-1} / c_{j+1})
  double* vs = va + VB_MAX_NI;                        // scaled operand of an FP32 product
  double* vx = vs + VB_MAX_NI;                        // x_j, or the backward operand
  double* vp = vx + VB_MAX_NI;                        // product D_j x_j
  double* vq = vp + VB_MAX_NI;                        // product Inv v
  const int tid = threadIdx.x;
  const bool own = tid < n;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
  }
  __syncthreads();
  // the inverse of layer j, FP32 or FP64
  auto inv_src = [&](int j) -> const void* {
    return f64 ? static_cast<const void*>(w.inv + (int64_t)j * n * ld)
               : static_cast<const void*>(mv.X + (int64_t)j * n * ldf);
  };
  // stage contents: forward step j = [D_j (refinement)] + [Inv_{j-1} (j > 0)];
  // backward step j = [Inv_j]
  auto issue = [&](int s, bool fwd, int j) {
    char* st = ring + (size_t)(s & 1) * sb;
    const bool with_d = fwd && !FIRST;
    const bool with_x = !fwd || j > 0;
    const uint32_t bytes = (with_d ? dbytes : 0u) + (with_x ? xbytes : 0u);
    mbar_expect_tx(&bars[s & 1], bytes);
    if (with_d) bulk_g2s(st + doff, w.inv + (int64_t)j * n * ld, dbytes, &bars[s & 1]);
    if (with_x) bulk_g2s(st + xoff, inv_src(fwd ? j - 1 : j), xbytes, &bars[s & 1]);
  };
  int issued = 0, waited = 0;   // stage counters (thread 0 issues; everyone waits)
  auto wait_stage = [&]() -> bool {
    const int s = waited;
    const bool ok = mbar_wait(&bars[s & 1], (uint32_t)((s >> 1) & 1), wlim);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        for (int s3 = s; s3 < issued; ++s3) mbar_wait(&bars[s3 & 1], (uint32_t)((s3 >> 1) & 1), WAIT_LIMIT);
        atomicOr(status + b, VB_STATUS_WATCHDOG);
      }
      return false;
    }
    ++waited;
    return true;
  };
  // product of the inverse held at stage offset xoff with r o v (FP32) or v (FP64)
  auto inv_apply = [&](const char* st, const double* rs_j, const double* v, double* out) {
    if (f64) {
      mx_matvec(reinterpret_cast<const double*>(st + xoff), n, ld, v, out);
    } else {
      if (own) vs[tid] = rs_j[tid] * v[tid];
      __syncthreads();
      mx_matvec(reinterpret_cast<const float*>(st + xoff), n, ldf, vs, out);
    }
  };

  // ---- forward: r_j = b_j - (M x)_j, r'_j = r_j - sub[j-1] o (Inv_{j-1} r'_{j-1})
  const int j0 = FIRST ? 1 : 0;   // FIRST: layer 0 needs no block
  const int F = nz - j0;          // forward stages
  if (FIRST && own) {
    const double r0 = bb[tid];
    va[tid] = r0;
    mv.tmp[tid] = r0;
  }
  if (tid == 0) {
    for (int q = 0; q < 2 && q < F; ++q) {
      issue(q, true, j0 + q);
      ++issued;
    }
  }
  for (int j = j0; j < nz; ++j) {
    const int s = j - j0;
    double xm = 0.0, xp = 0.0, bj = 0.0, cm = 0.0, cp = 0.0;
    if (own) {
      bj = bb[(int64_t)j * n + tid];
      cm = j > 0 ? w.subn[(int64_t)(j - 1) * n + tid] : 0.0;
      if (!FIRST) {
        vx[tid] = xb[(int64_t)j * n + tid];
        xm = j > 0 ? xb[(int64_t)(j - 1) * n + tid] : 0.0;
        xp = j < nz - 1 ? xb[(int64_t)(j + 1) * n + tid] : 0.0;
        cp = j < nz - 1 ? w.supn[(int64_t)j * n + tid] : 0.0;
      }
    }
    if (!wait_stage()) return;
    const char* st = ring + (size_t)(s & 1) * sb;
    if (!FIRST) mx_matvec(reinterpret_cast<const double*>(st + doff), n, ld, vx, vp);
    if (j > 0) inv_apply(st, mv.rs + (int64_t)(j - 1) * n, va, vq);
    __syncthreads();
    if (tid == 0 && issued < F) {
      fence_proxy_async();
      issue(issued, true, j0 + issued);
      ++issued;
    }
    if (own) {
      double r = bj;
      if (!FIRST) {
        double mx = vp[tid];
        if (j > 0) mx = mx + cm * xm;
        if (j < nz - 1) mx = mx + cp * xp;
        r = r - mx;
      }
      if (j > 0) r = r - cm * vq[tid];
      mv.tmp[(int64_t)j * n + tid] = r;
      va[tid] = r;
    }
    __syncthreads();
  }
  // ---- backward: c_j = Inv_j (r'_j - sup[j] o c_{j+1}); x_j += c_j (x_j = c_j on the first pass)
  //      stage F + q holds Inv_{nz-1-q}
  if (tid == 0) {
    fence_proxy_async();
    for (int q = 0; q < 2 && q < nz; ++q) {
      issue(F + q, false, nz - 1 - q);
      ++issued;
    }
  }
  double cmax = 0.0, xmax = 0.0;
  bool bad = false;
  for (int q = 0; q < nz; ++q) {
    const int j = nz - 1 - q;
    if (own) {
      double v = mv.tmp[(int64_t)j * n + tid];
      if (j < nz - 1) v = v - w.supn[(int64_t)j * n + tid] * va[tid];
      vx[tid] = v;
    }
    if (!wait_stage()) return;
    const char* st = ring + (size_t)((F + q) & 1) * sb;
    inv_apply(st, mv.rs + (int64_t)j * n, vx, vq);
    __syncthreads();
    if (tid == 0 && issued < F + nz) {
      fence_proxy_async();
      issue(issued, false, nz - 1 - (issued - F));
      ++issued;
    }
    if (own) {
      const double c = vq[tid];
      const double xn = FIRST ? c : xb[(int64_t)j * n + tid] + c;
      xb[(int64_t)j * n + tid] = xn;
      va[tid] = c;
      cmax = fmax(cmax, fabs(c));
      xmax = fmax(xmax, fabs(xn));
      bad |= !isfinite(xn);
    }
    __syncthreads();
  }
  // ---- convergence of this atmosphere
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, off));
    xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, off));
  }
  const int anybad = __any_sync(0xffffffffu, bad);
  if ((tid & 31) == 0) {
    red[tid >> 5][0] = cmax;
    red[tid >> 5][1] = xmax;
    redb[tid >> 5] = anybad;
  }
  __syncthreads();
  if (tid == 0) {
    double cm2 = red[0][0], xm2 = red[0][1];
    int nb = redb[0];
    for (int q = 1; q < MX_THREADS / 32; ++q) {
      cm2 = fmax(cm2, red[q][0]);
      xm2 = fmax(xm2, red[q][1]);
      nb |= redb[q];
    }
    if (passes) passes[b] += 1;
    if (FIRST) {
      if (md != MX_FP64) mode[b] = MX_REFINE;
    } else if (!nb && cm2 <= tol * xm2) {
      mode[b] = MX_DONE;
    }
  }
}

// Mode bookkeeping between the passes (one thread per atmosphere):
//  op 0 (after the FP32 factor): an FP32 zero pivot, non-finite inverse or
//        watchdog sends the atmosphere to MX_FP64 (todo = 1); status32 is
//        cleared.
//  op 1 (after the refinement passes): MX_REFINE atmospheres stalled: to
//        MX_FP64 with VB_STATUS_REFINE_STALL (todo = 1); others todo = 0.
__global__ void mx_mode_kernel(int batch, int op, int32_t* __restrict__ mode, int32_t* __restrict__ todo,
                               int32_t* __restrict__ status32, int32_t* __restrict__ status) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  int t = 0;
  if (op == 0) {
    const bool failed = (status32[b] & (VB_STATUS_ZERO_PIVOT | VB_STATUS_NONFINITE | VB_STATUS_WATCHDOG)) != 0;
    mode[b] = failed ? MX_FP64 : MX_REFINE;
    if (status32[b] & VB_STATUS_WATCHDOG) status[b] |= VB_STATUS_WATCHDOG;
    status32[b] = 0;
    t = failed;
  } else if (mode[b] == MX_REFINE) {
    mode[b] = MX_FP64;
    status[b] |= VB_STATUS_REFINE_STALL;
    t = 1;
  }
  todo[b] = t;
}

// sol = y + 3/(2r) k1 + 1/(2r) k2, delta = |sol - (y + k1/r)| (jax_step.py:313-314)
// from the refined stage vectors (k1 rows, k2 in the aux rows).
__global__ void mx_finish_kernel(Batch B, const double* __restrict__ ws, const double* __restrict__ y,
                                 double* __restrict__ sol, double* __restrict__ delta, int32_t* __restrict__ status) {
  const int b = blockIdx.y, j = blockIdx.x;
  const Geo g = geo_of(B, b);
  if (j >= g.nz) return;
  const int n = B.ni;
  WsView w = ws_view(const_cast<double*>(ws), g, n, B.ld);
  const double r = ros2_r();
  bool bad = false;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int64_t e = g.z0 * n + (int64_t)j * n + i;
    const double k1 = w.k1[(int64_t)j * n + i], k2 = w.aux[(int64_t)j * n + i], yv = y[e];
    const double s = yv + (3.0 / (2.0 * r)) * k1 + (1.0 / (2.0 * r)) * k2;
    const double yk2 = yv + k1 / r;
    sol[e] = s;
    delta[e] = fabs(s - yk2);
    bad |= !isfinite(s);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status + b, VB_STATUS_NONFINITE);
}

template <bool FIRST>
static cudaError_t launch_mx_pass_t(const Batch& B, double* ws, void* mxr, int xsel, int32_t* mode,
                                    const int32_t* only, int32_t* passes, double tol, int32_t* status,
                                    long long wlim, cudaStream_t st) {
  const size_t sm = mx_pass_smem(B.ni, !FIRST);
  cudaError_t e = cudaFuncSetAttribute(mx_pass_kernel<FIRST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  mx_pass_kernel<FIRST><<<B.count, MX_THREADS, sm, st>>>(B, ws, mxr, xsel, mode, only, passes, tol, status, wlim);
  return cudaGetLastError();
}

cudaError_t launch_mx_pass(const Batch& B, double* ws, void* mxr, int xsel, bool first, int32_t* mode,
                           const int32_t* only, int32_t* passes, double tol, int32_t* status, cudaStream_t st) {
  const long long wlim = wait_limit();
  return first ? launch_mx_pass_t<true>(B, ws, mxr, xsel, mode, only, passes, tol, status, wlim, st)
               : launch_mx_pass_t<false>(B, ws, mxr, xsel, mode, only, passes, tol, status, wlim, st);
}

cudaError_t launch_mx_mode(int batch, int op, int32_t* mode, int32_t* todo, int32_t* status32, int32_t* status,
                           cudaStream_t st) {
  mx_mode_kernel<<<(batch + 127) / 128, 128, 0, st>>>(batch, op, mode, todo, status32, status);
  return cudaGetLastError();
}

cudaError_t launch_mx_finish(const Batch& B, const double* ws, const double* y, double* sol, double* delta,
                             int32_t* status, cudaStream_t st) {
  dim3 grid(B.nz, B.count);
  mx_finish_kernel<<<grid, 128, 0, st>>>(B, ws, y, sol, delta, status);
  return cudaGetLastError();
}

}  // namespace vb
