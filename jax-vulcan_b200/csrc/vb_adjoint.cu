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

// ---- cotangents of every transport leaf of the atmosphere blob
// Fields of the blob in VB_ATM_DOUBLES order that the diffusion depends on.
enum AtmField { F_KZZ, F_DZI, F_VZ, F_HPI, F_TI, F_TCO, F_G, F_DZZ, F_VM, F_VS, F_MS, F_ALPHA, F_TOP, F_BOT,
                F_VDEP, N_FIELDS };

// Reads of an atmosphere as Duals with the derivative seeded on one element
// (field f, flat element e of that field).
struct SeedAcc {
  AtmRef a;
  int ni, f;
  int64_t e;
  __device__ Dual s(int fld, int64_t idx, double v) const { return {v, (fld == f && idx == e) ? 1.0 : 0.0}; }
  __device__ Dual Kzz(int m) const { return s(F_KZZ, m, a.Kzz[m]); }
  __device__ Dual dzi(int m) const { return s(F_DZI, m, a.dzi[m]); }
  __device__ Dual vz(int m) const { return s(F_VZ, m, a.vz[m]); }
  __device__ Dual Hpi(int m) const { return s(F_HPI, m, a.Hpi[m]); }
  __device__ Dual Ti(int m) const { return s(F_TI, m, a.Ti[m]); }
  __device__ Dual Tco(int m) const { return s(F_TCO, m, a.Tco[m]); }
  __device__ Dual g(int m) const { return s(F_G, m, a.g[m]); }
  __device__ Dual Dzz(int m, int i) const { return s(F_DZZ, (int64_t)m * ni + i, a.Dzz[(int64_t)m * ni + i]); }
  __device__ Dual vm(int m, int i) const { return s(F_VM, (int64_t)m * ni + i, a.vm[(int64_t)m * ni + i]); }
  __device__ Dual vs(int m, int i) const { return s(F_VS, (int64_t)m * ni + i, a.vs[(int64_t)m * ni + i]); }
  __device__ Dual ms(int i) const { return s(F_MS, i, a.ms[i]); }
  __device__ Dual alpha(int i) const { return s(F_ALPHA, i, a.alpha[i]); }
  __device__ Dual top(int i) const { return s(F_TOP, i, a.top[i]); }
  __device__ Dual bot(int i) const { return s(F_BOT, i, a.bot[i]); }
  __device__ Dual vdep(int i) const { return s(F_VDEP, i, a.vdep[i]); }
};

// diff[j][i] with boundary fluxes (jax_step.py:223-246), the terms of the
// forward kernels' layer_diffusion, as a Dual.
__device__ inline Dual diff_entry(const SeedAcc& acc, const double* yb, double ysm, double ys0, double ysp, int nz,
                                  int ni, int j, int i, int flags) {
  const double use_vm = (flags & VB_USE_VM_MOL) ? 1.0 : 0.0;
  const double use_set = (flags & VB_USE_SETTLING) ? 1.0 : 0.0;
  Dual Ae, Be, Ce, Am, Bm, Cm;
  eddy_row_t<Dual>(acc, nz, j, ysm, ys0, ysp, Ae, Be, Ce);
  mol_row_t<Dual>(acc, nz, j, i, ysm, ys0, ysp, use_vm, use_set, Am, Bm, Cm);
  const Dual At = Ae + Am, Bt = Be + Bm, Ct = Ce + Cm;
  const double y0 = yb[(int64_t)j * ni + i];
  Dual d;
  if (j == 0) {
    d = At * y0 + Bt * yb[(int64_t)(j + 1) * ni + i];
  } else if (j == nz - 1) {
    d = At * y0 + Ct * yb[(int64_t)(j - 1) * ni + i];
  } else {
    d = At * y0 + Bt * yb[(int64_t)(j + 1) * ni + i] + Ct * yb[(int64_t)(j - 1) * ni + i];
  }
  if (j == nz - 1 && (flags & VB_USE_TOPFLUX)) d = d + acc.top(i) / acc.dzi(nz - 2);
  if (j == 0 && (flags & VB_USE_BOTFLUX)) d = d + (acc.bot(i) - y0 * acc.vdep(i)) / acc.dzi(0);
  return d;
}

// One thread per leaf element: g = -sum over the stencil rows (and species)
// the element enters of lambda . d diff / d leaf, written at the element's
// place in the cotangent blob. Grid: (element blocks, atmospheres).
__global__ void __launch_bounds__(128)
vjp_atm_kernel(Batch B, const double* __restrict__ y, const double* __restrict__ atm, int flags,
               const double* __restrict__ lam, double* __restrict__ g_atm) {
  const int b = blockIdx.y;
  const Geo g = geo_of(B, b);
  const int ni = B.ni, nz = g.nz;
  const int64_t NI = ni, NZ = nz;
  const int64_t cnt[N_FIELDS] = {NZ - 1, NZ - 1, NZ - 1, NZ - 1, NZ - 1, NZ, NZ, (NZ - 1) * NI, NZ * NI,
                                 (NZ - 1) * NI, NI, NI, NI, NI, NI};
  int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int f = 0;
  while (f < N_FIELDS && q >= cnt[f]) q -= cnt[f++];
  if (f >= N_FIELDS) return;
  const double* blob = atm + g.atm;
  SeedAcc acc{atm_ref(blob, nz, ni), ni, f, q};
  const double* yb = y + g.z0 * ni;
  const double* lb = lam + g.z0 * ni;
  int lo = 0, hi = nz - 1, i0 = 0, i1 = ni - 1;
  if (f <= F_TI) { lo = (int)q - 1; hi = (int)q + 2; }                           // interface m = q
  else if (f == F_TCO || f == F_G) { lo = (int)q - 1; hi = (int)q + 1; }          // layer q
  else if (f == F_DZZ || f == F_VS) { const int m = (int)(q / ni); i0 = i1 = (int)(q % ni); lo = m - 1; hi = m + 2; }
  else if (f == F_VM) { const int l = (int)(q / ni); i0 = i1 = (int)(q % ni); lo = l - 1; hi = l + 1; }
  else if (f == F_MS || f == F_ALPHA) { i0 = i1 = (int)q; }
  else if (f == F_TOP) { i0 = i1 = (int)q; lo = hi = nz - 1; }
  else { i0 = i1 = (int)q; lo = hi = 0; }                                         // bot_flux, bot_vdep
  lo = max(lo, 0);
  hi = min(hi, nz - 1);
  double gsum = 0.0;
  for (int j = lo; j <= hi; ++j) {
    // gas sums of rows j-1, j, j+1 (0 outside the column, as the forward kernels)
    double ys3[3];
    for (int w = 0; w < 3; ++w) {
      const int jj = j - 1 + w;
      ys3[w] = (jj >= 0 && jj < nz) ? pairwise_sum_masked(yb + (int64_t)jj * ni, acc.a.gas, ni) : 0.0;
    }
    for (int i = i0; i <= i1; ++i) {
      const Dual d = diff_entry(acc, yb, ys3[0], ys3[1], ys3[2], nz, ni, j, i, flags);
      gsum += lb[(int64_t)j * ni + i] * d.d;
    }
  }
  const AtmOff o = atm_offsets(nz, ni);
  const int64_t field_off[N_FIELDS] = {o.Kzz, o.dzi, o.vz, o.Hpi, o.Ti, o.Tco, o.g, o.Dzz, o.vm, o.vs,
                                       o.ms, o.alpha, o.top, o.bot, o.vdep};
  g_atm[g.atm + field_off[f] + q] = -gsum;
}

// Copy the workspace's first-stage rows (k1: the adjoint's lambda, or the
// Ros2 step's k1) and, with k2 != nullptr, the Ros2 step's second-stage rows
// (kept in the aux rows by the final back sweep) into [layers][ni] arrays.
__global__ void gather_stages_kernel(Batch B, const double* __restrict__ ws, double* __restrict__ k1,
                                     double* __restrict__ k2) {
  const int b = blockIdx.y, j = blockIdx.x;
  Geo g = geo_of(B, b);
  if (j >= g.nz) return;
  WsView w = ws_view(const_cast<double*>(ws), g, B.ni, B.ld);
  const int64_t src = (int64_t)j * B.ni, dst = g.z0 * B.ni + (int64_t)j * B.ni;
  for (int i = threadIdx.x; i < B.ni; i += blockDim.x) {
    if (k1) k1[dst + i] = w.k1[src + i];
    if (k2) k2[dst + i] = w.aux[src + i];
  }
}

cudaError_t launch_gather_stages(const Batch& B, const double* ws, double* k1, double* k2, cudaStream_t st) {
  if (!k1 && !k2) return cudaSuccess;
  dim3 grid(B.nz, B.count);
  gather_stages_kernel<<<grid, 128, 0, st>>>(B, ws, k1, k2);
  return cudaGetLastError();
}

cudaError_t launch_vjp_atm(const Batch& B, const double* y, const double* atm, int flags, const double* lam,
                           double* g_atm, cudaStream_t st) {
  const int64_t NZ = B.nz, NI = B.ni;
  const int64_t per = 5 * (NZ - 1) + 2 * NZ + 2 * (NZ - 1) * NI + NZ * NI + 5 * NI;
  dim3 grid((unsigned)((per + 127) / 128), B.count);
  vjp_atm_kernel<<<grid, 128, 0, st>>>(B, y, atm, flags, lam, g_atm);
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
