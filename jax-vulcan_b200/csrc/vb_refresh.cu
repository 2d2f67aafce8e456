// Atmosphere refresh and condensation (reference atm_refresh.py, conden.py).
//
// refresh_kernel (CTA per atmosphere; inside the loop, only the atmospheres
//   whose taken attempt falls on the refresh cadence): mean molecular mass per layer, then
//   the hydrostatic integration, a true serial recurrence in z
//   (zco[j+1] = zco[j] + dz[j]), run by one thread upward from the reference
//   layer and downward below it; the interface means and the escape fluxes
//   in parallel; g, dzi, Hpi and the escape entries of top_flux are spliced
//   into the atmosphere blob.
// conden_rates_kernel (thread per layer x reaction): condensation and
//   evaporation rows of k.
// relax_kernel (CTA per atmosphere, warp per layer): the implicit-Euler
//   cold-trap relaxation of one species and the re-projection of y.
// Compiled with --fmad=false: products and sums round as the reference's
// element-wise expressions do.
#include <cuda_runtime.h>

#include "vb_common.cuh"
#include "vb_launch.cuh"
#include "vb_layer.cuh"

namespace vb {

constexpr int REFRESH_THREADS = 128;
constexpr int RELAX_THREADS = 256;

__global__ void __launch_bounds__(REFRESH_THREADS)
refresh_kernel(int nz, int ni, VbRefreshParams p, const double* __restrict__ pico, const double* __restrict__ mol_mass,
               const int32_t* __restrict__ esc, const double* __restrict__ y, const double* __restrict__ ymix,
               double* __restrict__ atm, double* __restrict__ mu_o, double* __restrict__ Hp_o,
               double* __restrict__ dz_o, double* __restrict__ zco_o, const VbLoopScalars* __restrict__ st,
               int update_frq, const VbConvState* __restrict__ conv) {
  extern __shared__ double sm[];
  if (st) {   // inside the loop: taken attempts on the refresh cadence only (outer_loop.py:813-818)
    const VbLoopScalars s = st[blockIdx.x];
    const bool done = conv && conv[blockIdx.x].done;
    if (done || s.last_decision == 0 || (s.accept_count - 1) % update_frq != 0) return;
  }
  double* mu = sm;            // [nz]
  double* g = mu + nz;        // [nz]
  double* Hp = g + nz;        // [nz]
  double* dz = Hp + nz;       // [nz]
  double* zco = dz + nz;      // [nz+1]
  const int b = blockIdx.x;
  const AtmOff off = atm_offsets(nz, ni);
  double* A = atm + (int64_t)b * VB_ATM_DOUBLES(nz, ni);
  const double* T = A + off.Tco;
  const double* pc = pico + (int64_t)b * (nz + 1);
  const double* xb = ymix + (int64_t)b * nz * ni;
  for (int j = threadIdx.x; j < nz; j += blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < ni; ++i) s = s + xb[(int64_t)j * ni + i] * mol_mass[i];
    mu[j] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {   // atm_refresh.py:57-96
    const int pref = p.pref_indx;
    double z = p.zco_pref;
    zco[pref] = z;
    for (int i = pref; i < nz; ++i) {
      double gi = p.gs;
      if (i != pref) {
        const double q = p.Rp / (p.Rp + z);
        gi = p.gs * (q * q);
      }
      const double h = p.kb * T[i] / (mu[i] / p.Navo * gi);
      const double d = h * log(pc[i] / pc[i + 1]);
      z = z + d;
      g[i] = gi; Hp[i] = h; dz[i] = d; zco[i + 1] = z;
    }
    z = p.zco_pref;
    for (int i = pref - 1; i >= 0; --i) {
      const double q = p.Rp / (p.Rp + z);
      const double gi = p.gs * (q * q);
      const double h = p.kb * T[i] / (mu[i] / p.Navo * gi);
      const double d = h * log(pc[i] / pc[i + 1]);
      z = z - d;
      g[i] = gi; Hp[i] = h; dz[i] = d; zco[i] = z;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nz; j += blockDim.x) {
    A[off.g + j] = g[j];
    if (j < nz - 1) {
      A[off.dzi + j] = 0.5 * (dz[j] + dz[j + 1]);
      A[off.Hpi + j] = 0.5 * (Hp[j] + Hp[j + 1]);
    }
    if (mu_o) mu_o[(int64_t)b * nz + j] = mu[j];
    if (Hp_o) Hp_o[(int64_t)b * nz + j] = Hp[j];
    if (dz_o) dz_o[(int64_t)b * nz + j] = dz[j];
  }
  if (zco_o)
    for (int j = threadIdx.x; j <= nz; j += blockDim.x) zco_o[(int64_t)b * (nz + 1) + j] = zco[j];
  // atm_refresh.py:103-122
  const double* ytop = y + ((int64_t)b * nz + nz - 1) * ni;
  for (int e = threadIdx.x; e < p.n_esc; e += blockDim.x) {
    const int sp = esc[e];
    const double Dz = A[off.Dzz + (int64_t)(nz - 2) * ni + sp];
    double f = -Dz * ytop[sp] * (1.0 / Hp[nz - 1] - A[off.ms + sp] * g[nz - 1] / (p.Navo * p.kb * T[nz - 1]));
    f = (f != f) ? f : fmax(f, -p.max_flux);
    A[off.top + sp] = f;
  }
}

__global__ void conden_rates_kernel(int nz, int ni, int nr, int n_re, const int32_t* __restrict__ re_idx,
                                    const int32_t* __restrict__ sp_idx, const double* __restrict__ coeff,
                                    const double* __restrict__ Dg, const double* __restrict__ sat,
                                    const double* __restrict__ y, double* __restrict__ k) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y, b = blockIdx.z;
  if (z >= nz) return;
  const int64_t o = ((int64_t)b * n_re + r) * nz + z;
  const double rate = Dg[o] * coeff[r] * (y[((int64_t)b * nz + z) * ni + sp_idx[r]] - sat[o]);
  const double pos = (rate != rate) ? rate : fmax(rate, 0.0);
  const double neg = (rate != rate) ? rate : fmax(-rate, 0.0);
  double* kb = k + (int64_t)b * (nr + 1) * nz;
  kb[(int64_t)re_idx[r] * nz + z] = pos;
  kb[(int64_t)(re_idx[r] + 1) * nz + z] = neg;
}

// One layer of the cold-trap relaxation of one species (conden.py:74-160),
// by one warp: lane 0 forms the scalar updates of the species and its
// condensate, every lane re-projects y = ymix * (gas sum of y before the
// update) over the row.
__device__ inline void relax_layer(int lane, int j, int ni, const VbRelaxParams& p, double Dg, double s, double n0,
                                   const double* gasm, double dt, double* yr, double* xr) {
  const int sp = p.sp, ls = p.sp_l_s;
  double ysum = 0.0, x_sp = 0.0, x_ls = 0.0;
  if (lane == 0) {
    ysum = pairwise_sum_masked(yr, gasm, ni);
    double denom = Dg * p.m_over_rho_r2 * (yr[sp] - s);
    if (fabs(denom) < 1e-300) denom = 1e-300;
    const double tau = 1.0 / denom;
    const double sat_mix = s / n0;
    const double y_conden = (xr[sp] + dt / tau * sat_mix) / (1.0 + dt / tau);
    double ice = (yr[sp] - s) * dt / tau;
    ice = fmin(yr[ls], ice);
    bool conden = tau > 0.0;
    if (p.conden_top >= 0) conden = conden && (j <= p.conden_top);
    const double dc = conden ? xr[sp] - y_conden : 0.0;
    const double de = tau < 0.0 ? ice / n0 : 0.0;
    x_ls = xr[ls] + dc;
    x_sp = xr[sp] + (-dc);
    x_sp = x_sp + de;
    x_ls = x_ls + (-de);
    if (p.conden_top >= 0) x_ls = fmax(x_ls, 0.0);
  }
  ysum = __shfl_sync(0xffffffffu, ysum, 0);
  x_sp = __shfl_sync(0xffffffffu, x_sp, 0);
  x_ls = __shfl_sync(0xffffffffu, x_ls, 0);
  for (int i = lane; i < ni; i += 32) {
    double x = xr[i];
    if (i == sp) x = x_sp;
    if (i == ls) x = x_ls;
    xr[i] = x;
    yr[i] = x * ysum;
  }
  __syncwarp();
}

__global__ void __launch_bounds__(RELAX_THREADS)
relax_kernel(int nz, int ni, VbRelaxParams p, const double* __restrict__ Dg, const double* __restrict__ sat,
             const double* __restrict__ atm, const double* __restrict__ dtp, double* __restrict__ y,
             double* __restrict__ ymix) {
  const int b = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const AtmOff off = atm_offsets(nz, ni);
  const double* A = atm + (int64_t)b * VB_ATM_DOUBLES(nz, ni);
  const double dt = dtp[b];
  for (int j = warp; j < nz; j += RELAX_THREADS / 32)
    relax_layer(lane, j, ni, p, Dg[(int64_t)b * nz + j], sat[(int64_t)b * nz + j], A[off.M + j], A + off.gas, dt,
                y + ((int64_t)b * nz + j) * ni, ymix + ((int64_t)b * nz + j) * ni);
}

// Condensation inside the adaptive loop (outer_loop.py:770-800), CTA per
// atmosphere: the condensation rows of k from the attempt's clipped state,
// the H2O and NH3 relaxations of that state with the attempt's dt, and for
// an accepted attempt the hydrostatic rebalance of the body redone from the
// relaxed state (the same per-element expressions as loop_body_kernel).
__global__ void __launch_bounds__(RELAX_THREADS)
loop_condense_kernel(int nz, int ni, int nr, VbCondenLoop c, VbLoopParams p, const double* __restrict__ atm,
                     const uint8_t* __restrict__ gas, const double* __restrict__ compo,
                     const double* __restrict__ atom_ini, const VbLoopScalars* __restrict__ st,
                     const VbConvState* __restrict__ conv, const double* __restrict__ pre_td,
                     double* __restrict__ pre_y, double* __restrict__ pre_ymix,
                     double* y, double* y_prev, double* ymix,   // may alias one another (y == y_prev)
                     double* __restrict__ atom_loss, double* __restrict__ atom_loss_prev, double* __restrict__ k) {
  constexpr int W = RELAX_THREADS / 32;
  __shared__ double red[W][VB_LOOP_MAX_ATOMS];
  const int b = blockIdx.x;
  if (conv && conv[b].done) return;                                   // the body left it alone
  const int dec = st[b].last_decision;
  if (dec == 0 || !(pre_td[2 * (int64_t)b] >= c.start_conden_time)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const AtmOff off = atm_offsets(nz, ni);
  const double* A = atm + (int64_t)b * VB_ATM_DOUBLES(nz, ni);
  const double* M = A + off.M;
  const double dt = pre_td[2 * (int64_t)b + 1];
  double* py = pre_y + (int64_t)b * nz * ni;
  double* px = pre_ymix + (int64_t)b * nz * ni;
  // condensation rows of k (conden.py:55-71) from the clipped state
  double* kb = k + (int64_t)b * (nr + 1) * nz;
  for (int e = threadIdx.x; e < c.n_re * nz; e += RELAX_THREADS) {
    const int r = e / nz, z = e - r * nz;
    const int64_t o = ((int64_t)b * c.n_re + r) * nz + z;
    const double rate = c.Dg_re[o] * c.coeff[r] * (py[(int64_t)z * ni + c.sp_idx[r]] - c.sat_re[o]);
    kb[(int64_t)c.re_idx[r] * nz + z] = (rate != rate) ? rate : fmax(rate, 0.0);
    kb[(int64_t)(c.re_idx[r] + 1) * nz + z] = (rate != rate) ? rate : fmax(-rate, 0.0);
  }
  __syncthreads();   // the rates read the clipped state before the relaxation rewrites it
  // H2O, then NH3 (conden.py:74-160)
  for (int j = warp; j < nz; j += W) {
    double* yr = py + (int64_t)j * ni;
    double* xr = px + (int64_t)j * ni;
    if (c.h2o_active) {
      VbRelaxParams q{c.h2o_sp, c.h2o_l_s, -1, 0, c.h2o_m_over_rho_r2};
      relax_layer(lane, j, ni, q, c.h2o_Dg[(int64_t)b * nz + j], c.h2o_sat[(int64_t)b * nz + j], M[j], A + off.gas,
                  dt, yr, xr);
    }
    if (c.nh3_active) {
      VbRelaxParams q{c.nh3_sp, c.nh3_l_s, c.nh3_conden_top, 0, c.nh3_m_over_rho_r2};
      relax_layer(lane, j, ni, q, c.nh3_Dg[(int64_t)b * nz + j], c.nh3_sat[(int64_t)b * nz + j], M[j], A + off.gas,
                  dt, yr, xr);
    }
  }
  if (dec != 1) return;   // a force-accepted attempt keeps y_prev (outer_loop.py:903-906)
  __syncthreads();
  // hydrostatic rebalance from the relaxed state (outer_loop.py:846-853, 899-917)
  const bool hydro = (p.flags & VB_LOOP_HYDRO_PARTIAL) != 0;
  const int na = p.n_atoms;
  double pb[VB_LOOP_MAX_ATOMS];
#pragma unroll
  for (int a = 0; a < VB_LOOP_MAX_ATOMS; ++a) pb[a] = 0.0;
  double* yb = y + (int64_t)b * nz * ni;
  double* ypb = y_prev + (int64_t)b * nz * ni;
  double* xb = ymix + (int64_t)b * nz * ni;
  for (int j = warp; j < nz; j += W) {
    double bs = 0.0;
    for (int i = lane; i < ni; i += 32) {
      const bool gi = !gas || gas[i];
      const double bv = (hydro && !gi) ? py[(int64_t)j * ni + i] : M[j] * px[(int64_t)j * ni + i];
      if (gi) bs += bv;
      yb[(int64_t)j * ni + i] = bv;
      ypb[(int64_t)j * ni + i] = bv;
#pragma unroll
      for (int a = 0; a < VB_LOOP_MAX_ATOMS; ++a)
        if (a < na) pb[a] += compo[i * na + a] * bv;
    }
#pragma unroll
    for (int off2 = 16; off2 > 0; off2 >>= 1) bs += __shfl_xor_sync(0xffffffffu, bs, off2);
    __syncwarp();
    for (int i = lane; i < ni; i += 32) xb[(int64_t)j * ni + i] = yb[(int64_t)j * ni + i] / bs;
  }
#pragma unroll
  for (int a = 0; a < VB_LOOP_MAX_ATOMS; ++a) {
    if (a < na) {
#pragma unroll
      for (int off2 = 16; off2 > 0; off2 >>= 1) pb[a] += __shfl_xor_sync(0xffffffffu, pb[a], off2);
    }
  }
  if (lane == 0)
    for (int a = 0; a < na; ++a) red[warp][a] = pb[a];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int a = 0; a < na; ++a) {
      double sb = red[0][a];
      for (int w = 1; w < W; ++w) sb += red[w][a];
      const double ini = atom_ini[(int64_t)b * na + a];
      const double al = (sb - ini) / ini;
      atom_loss[(int64_t)b * na + a] = al;
      atom_loss_prev[(int64_t)b * na + a] = al;
    }
  }
}

cudaError_t launch_atm_refresh(int batch, int nz, int ni, const VbRefreshParams& p, const double* pico,
                               const double* mol_mass, const int32_t* esc, const double* y, const double* ymix,
                               double* atm, double* mu, double* Hp, double* dz, double* zco,
                               const VbLoopScalars* loop_st, int update_frq, const VbConvState* conv,
                               cudaStream_t st) {
  const size_t smem = (5 * (size_t)nz + 1) * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(refresh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  refresh_kernel<<<batch, REFRESH_THREADS, smem, st>>>(nz, ni, p, pico, mol_mass, esc, y, ymix, atm, mu, Hp, dz, zco,
                                                       loop_st, update_frq, conv);
  return cudaGetLastError();
}

cudaError_t launch_conden_rates(int batch, int nz, int ni, int nr, int n_re, const int32_t* re_idx,
                                const int32_t* sp_idx, const double* coeff, const double* Dg, const double* sat,
                                const double* y, double* k, cudaStream_t st) {
  dim3 grid((nz + 127) / 128, n_re, batch);
  conden_rates_kernel<<<grid, 128, 0, st>>>(nz, ni, nr, n_re, re_idx, sp_idx, coeff, Dg, sat, y, k);
  return cudaGetLastError();
}

cudaError_t launch_conden_relax(int batch, int nz, int ni, const VbRelaxParams& p, const double* Dg,
                                const double* sat, const double* atm, const double* dt, double* y, double* ymix,
                                cudaStream_t st) {
  relax_kernel<<<batch, RELAX_THREADS, 0, st>>>(nz, ni, p, Dg, sat, atm, dt, y, ymix);
  return cudaGetLastError();
}

}  // namespace vb

namespace vb {
cudaError_t launch_loop_condense(int batch, int nz, int ni, int nr, const VbCondenLoop& c, const VbLoopParams& p,
                                 const double* atm, const uint8_t* gas, const double* compo, const double* atom_ini,
                                 const VbLoopScalars* st, const VbConvState* conv, const double* pre_td,
                                 double* pre_y, double* pre_ymix, double* y, double* y_prev, double* ymix,
                                 double* atom_loss, double* atom_loss_prev, double* k, cudaStream_t stream) {
  loop_condense_kernel<<<batch, RELAX_THREADS, 0, stream>>>(nz, ni, nr, c, p, atm, gas, compo, atom_ini, st, conv,
                                                            pre_td, pre_y, pre_ymix, y, y_prev, ymix, atom_loss,
                                                            atom_loss_prev, k);
  return cudaGetLastError();
}
}  // namespace vb
