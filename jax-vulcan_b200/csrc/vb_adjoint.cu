// VJP kernels of the implicit steady-state adjoint (reference
// steady_state_grad.py:214-233, 306-327): given lambda = J_y^{-T} v, the
// cotangents  cot = -lambda . df/dtheta  of the residual
// f = chem_rhs(y, M, k) + diffusion(y) (steady_state_grad.py:116-130) for
//   k[r, z]    (chem.py:92-125; f is linear in k),
//   M[z]       (three-body rates),
//   Kzz[m]     (eddy diffusion of the two layers sharing interface m,
//               jax_step.py:167-189),
//   top_flux, bot_flux, bot_vdep (boundary fluxes, jax_step.py:236-245).
#include <cuda_runtime.h>

#include "vb_common.cuh"
#include "vb_launch.cuh"
#include "vb_layer.cuh"

namespace vb {

constexpr int VJP_THREADS = 256;

// One CTA per (layer, atmosphere): g_k[r][z] = -P'[r] * S[r] with P' the rate
// per unit k and S = sum_s p_st lambda[p_idx] - sum_s r_st lambda[r_idx].
__global__ void __launch_bounds__(VJP_THREADS)
vjp_k_kernel(NetDev net, Batch B, const double* __restrict__ y, const double* __restrict__ k,
             const double* __restrict__ atm, double* __restrict__ ws, double* __restrict__ g_k,
             double* __restrict__ g_M) {
  __shared__ double ys[VB_MAX_NI + 1], ls[VB_MAX_NI + 1], red[VJP_THREADS / 32];
  const int b = blockIdx.y, j = blockIdx.x;
  Geo g = geo_of(B, b);
  if (j >= g.nz) return;
  const int ni = B.ni, nz = g.nz, T = net.T;
  AtmRef a = atm_ref(atm + g.atm, nz, ni);
  const double* lam = ws_view(ws, g, ni, B.ld).k1;   // lambda, [nz][ni]
  for (int i = threadIdx.x; i <= ni; i += blockDim.x) {
    ys[i] = i < ni ? y[g.z0 * ni + (int64_t)j * ni + i] : 1.0;
    ls[i] = i < ni ? lam[(int64_t)j * ni + i] : 0.0;
  }
  __syncthreads();
  const double M = a.M[j];
  const double* kc = k + g.z0 * (B.nr + 1) + j;
  double gm = 0.0;
  for (int r = threadIdx.x; r <= net.nr; r += blockDim.x) {
    double prod = 1.0, S = 0.0;
    for (int s = 0; s < T; ++s) {
      const double st = net.r_st[r * T + s];
      if (st > 0.0) prod = prod * pow_st(ys[net.r_idx[r * T + s]], st);
      S = S - st * ls[net.r_idx[r * T + s]];
      S = S + net.p_st[r * T + s] * ls[net.p_idx[r * T + s]];
    }
    const bool three = net.three[r] != 0;
    const double Pp = three ? prod * M : prod;
    if (g_k) g_k[g.z0 * (B.nr + 1) + (int64_t)r * nz + j] = -Pp * S;
    if (three) gm = gm - kc[(int64_t)r * nz] * prod * S;
  }
  if (g_M) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) gm += __shfl_xor_sync(0xffffffffu, gm, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = gm;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < VJP_THREADS / 32; ++w) t += red[w];
      g_M[g.z0 + j] = t;
    }
  }
}

// One CTA per atmosphere: eddy Kzz and boundary-flux cotangents.
__global__ void __launch_bounds__(VJP_THREADS)
vjp_transport_kernel(Batch B, const double* __restrict__ y, const double* __restrict__ atm, int flags,
                     double* __restrict__ ws, double* __restrict__ g_Kzz, double* __restrict__ g_top,
                     double* __restrict__ g_bot, double* __restrict__ g_vdep) {
  extern __shared__ double ysum[];
  const int b = blockIdx.x;
  Geo g = geo_of(B, b);
  const int ni = B.ni, nz = g.nz;
  AtmRef a = atm_ref(atm + g.atm, nz, ni);
  const double* yb = y + g.z0 * ni;
  const double* lb = ws_view(ws, g, ni, B.ld).k1;
  for (int j = threadIdx.x; j < nz; j += blockDim.x) ysum[j] = pairwise_sum_masked(yb + (int64_t)j * ni, a.gas, ni);
  __syncthreads();
  // stencil-row spacing h_j: dz_ave inside, dzi at the two boundary rows
  auto h_of = [&](int j) {
    if (j == 0) return a.dzi[0];
    if (j == nz - 1) return a.dzi[nz - 2];
    return 0.5 * (a.dzi[j - 1] + a.dzi[j]);
  };
  if (g_Kzz) {
    for (int m = threadIdx.x; m < nz - 1; m += blockDim.x) {
      const double h0 = h_of(m), h1 = h_of(m + 1);
      const double ys0 = ysum[m], ys1 = ysum[m + 1];
      double dLdF = 0.0;
      for (int i = 0; i < ni; ++i) {
        const double grad = yb[(int64_t)(m + 1) * ni + i] / ys1 - yb[(int64_t)m * ni + i] / ys0;
        dLdF += grad * (lb[(int64_t)m * ni + i] / h0 - lb[(int64_t)(m + 1) * ni + i] / h1);
      }
      g_Kzz[g.z0 + m] = -dLdF * (ys1 + ys0) / (2.0 * a.dzi[m]);
    }
  }
  for (int i = threadIdx.x; i < ni; i += blockDim.x) {
    const int64_t o = (int64_t)b * ni + i;
    if (g_top) g_top[o] = (flags & VB_USE_TOPFLUX) ? -lb[(int64_t)(nz - 1) * ni + i] / a.dzi[nz - 2] : 0.0;
    if (g_bot) g_bot[o] = (flags & VB_USE_BOTFLUX) ? -lb[i] / a.dzi[0] : 0.0;
    if (g_vdep) g_vdep[o] = (flags & VB_USE_BOTFLUX) ? lb[i] * yb[i] / a.dzi[0] : 0.0;
  }
}

__global__ void gather_k1_kernel(Batch B, double* __restrict__ ws, double* __restrict__ out) {
  const int b = blockIdx.y, j = blockIdx.x;
  Geo g = geo_of(B, b);
  if (j >= g.nz) return;
  const double* src = ws_view(ws, g, B.ni, B.ld).k1 + (int64_t)j * B.ni;
  for (int i = threadIdx.x; i < B.ni; i += blockDim.x) out[g.z0 * B.ni + (int64_t)j * B.ni + i] = src[i];
}

cudaError_t launch_gather_k1(const Batch& B, double* ws, double* out, cudaStream_t st) {
  if (!out) return cudaSuccess;
  dim3 grid(B.nz, B.count);
  gather_k1_kernel<<<grid, 128, 0, st>>>(B, ws, out);
  return cudaGetLastError();
}

cudaError_t launch_vjp(const NetDev& net, const Batch& B, const double* y, const double* k, const double* atm,
                       int flags, double* ws, double* g_k, double* g_M, double* g_Kzz, double* g_top,
                       double* g_bot, double* g_vdep, cudaStream_t st) {
  if (g_k || g_M) {
    dim3 grid(B.nz, B.count);
    vjp_k_kernel<<<grid, VJP_THREADS, 0, st>>>(net, B, y, k, atm, ws, g_k, g_M);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (g_Kzz || g_top || g_bot || g_vdep) {
    size_t sm = (size_t)B.nz * sizeof(double);
    vjp_transport_kernel<<<B.count, VJP_THREADS, sm, st>>>(B, y, atm, flags, ws, g_Kzz, g_top, g_bot, g_vdep);
    return cudaGetLastError();
  }
  return cudaSuccess;
}

}  // namespace vb
