// Per-layer chemistry and diffusion device code (compiled with --fmad=false so
// every product and sum is rounded exactly as the reference's NumPy/XLA
// element-wise expressions are; the operation order below mirrors the
// reference expressions term by term).
#pragma once
#include "vb_common.cuh"

namespace vb {

constexpr double KB = 1.38064852e-16;   // reference phy_const.py:3
constexpr double NAVO = 6.02214086e23;  // reference phy_const.py:4

// NumPy's pairwise summation of a contiguous row (the order np.sum uses for
// a reduction along a contiguous axis): 8 interleaved partial sums for
// 8 <= n <= 128, a plain loop below 8. Used for ysum (jax_step.py:161).
__device__ inline double pairwise_sum(const double* a, int n) {
  if (n < 8) {
    double r = 0.0;
    for (int i = 0; i < n; ++i) r = r + a[i];
    return r;
  }
  double r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = a[k];
  int i = 8;
  for (; i < n - (n % 8); i += 8) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = r[k] + a[i + k];
  }
  double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
  for (; i < n; ++i) res = res + a[i];
  return res;
}

// pairwise_sum of where(mask != 0, a, 0) without a staging copy.
__device__ inline double pairwise_sum_masked(const double* a, const double* mask, int n) {
  auto at = [&](int i) { return mask[i] != 0.0 ? a[i] : 0.0; };
  if (n < 8) {
    double r = 0.0;
    for (int i = 0; i < n; ++i) r = r + at(i);
    return r;
  }
  double r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = at(k);
  int i = 8;
  for (; i < n - (n % 8); i += 8) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = r[k] + at(i + k);
  }
  double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
  for (; i < n; ++i) res = res + at(i);
  return res;
}

// y**st as NumPy evaluates it for the integer stoichiometries of a network
// (st = 1, 2 exactly; other values through pow).
__device__ __forceinline__ double pow_st(double y, double st) {
  if (st == 1.0) return y;
  if (st == 2.0) return y * y;
  if (st == 0.0) return 1.0;
  return pow(y, st);
}

__device__ __forceinline__ double pos_part(double v) { return (v > 0.0 ? 1.0 : 0.0) * v; }
__device__ __forceinline__ double neg_part(double v) { return (v < 0.0 ? 1.0 : 0.0) * v; }

// Read-only view of one atmosphere's packed fields.
struct AtmRef {
  const double *Kzz, *dzi, *vz, *Hpi, *Ti, *Tco, *g, *M, *Dzz, *vm, *vs, *ms, *alpha, *top, *bot,
      *vdep, *gas;
};

__device__ __forceinline__ AtmRef atm_ref(const double* blob, int nz, int ni) {
  AtmOff o = atm_offsets(nz, ni);
  AtmRef a;
  a.Kzz = blob + o.Kzz; a.dzi = blob + o.dzi; a.vz = blob + o.vz; a.Hpi = blob + o.Hpi;
  a.Ti = blob + o.Ti; a.Tco = blob + o.Tco; a.g = blob + o.g; a.M = blob + o.M;
  a.Dzz = blob + o.Dzz; a.vm = blob + o.vm; a.vs = blob + o.vs; a.ms = blob + o.ms;
  a.alpha = blob + o.alpha; a.top = blob + o.top; a.bot = blob + o.bot; a.vdep = blob + o.vdep;
  a.gas = blob + o.gas;
  return a;
}

// Eddy coefficients of stencil row j (reference jax_step.py:167-193).
__device__ inline void eddy_row(const AtmRef& a, int nz, int j, double ysm, double ys0, double ysp,
                                double& A, double& Bc, double& C) {
  const double* Kzz = a.Kzz;
  const double* dzi = a.dzi;
  const double* vz = a.vz;
  if (j == 0) {
    A = -1.0 / dzi[0] * (Kzz[0] / dzi[0]) * (ysp + ys0) / 2.0 / ys0;
    A = A - pos_part(vz[0]) / dzi[0];
    Bc = 1.0 / dzi[0] * (Kzz[0] / dzi[0]) * (ysp + ys0) / 2.0 / ysp;
    Bc = Bc - neg_part(vz[0]) / dzi[0];
    C = 0.0;
  } else if (j == nz - 1) {
    int t = nz - 2;
    A = -1.0 / dzi[t] * (Kzz[t] / dzi[t]) * (ys0 + ysm) / 2.0 / ys0;
    A = A + neg_part(vz[t]) / dzi[t];
    C = 1.0 / dzi[t] * (Kzz[t] / dzi[t]) * (ys0 + ysm) / 2.0 / ysm;
    C = C + pos_part(vz[t]) / dzi[t];
    Bc = 0.0;
  } else {
    double dz_ave = 0.5 * (dzi[j - 1] + dzi[j]);
    A = -1.0 / dz_ave *
        (Kzz[j] / dzi[j] * (ysp + ys0) / 2.0 + Kzz[j - 1] / dzi[j - 1] * (ys0 + ysm) / 2.0) / ys0;
    Bc = 1.0 / dz_ave * Kzz[j] / dzi[j] * (ysp + ys0) / 2.0 / ysp;
    C = 1.0 / dz_ave * Kzz[j - 1] / dzi[j - 1] * (ys0 + ysm) / 2.0 / ysm;
    A = A - (pos_part(vz[j]) - neg_part(vz[j - 1])) / dz_ave;
    Bc = Bc - neg_part(vz[j]) / dz_ave;
    C = C + pos_part(vz[j - 1]) / dz_ave;
  }
}

// Gravity/thermal-diffusion factor of compute_diff_grav (jax_step.py:80-87):
// -1/Hpi[h] + ms*g[gi]/(Navo*kb*Ti[h]) + alpha/Ti[h]*(Tco[t1]-Tco[t0])/dzi[h].
__device__ __forceinline__ double grav_fac(const AtmRef& a, int i, int h, int gi, int t1, int t0) {
  return -1.0 / a.Hpi[h] + a.ms[i] * a.g[gi] / (NAVO * KB * a.Ti[h]) +
         a.alpha[i] / a.Ti[h] * (a.Tco[t1] - a.Tco[t0]) / a.dzi[h];
}

// Molecular-diffusion coefficients of species i on stencil row j, including the
// y-independent gravity / vm / settling pieces (jax_step.py:67-147, 195-218).
__device__ inline void mol_row(const AtmRef& a, int nz, int ni, int j, int i, double ysm, double ys0,
                               double ysp, double use_vm, double use_set, double& A, double& Bc,
                               double& C) {
  const double* dzi = a.dzi;
  if (j == 0) {
    double D0 = a.Dzz[i];
    double g0 = 1.0 / dzi[0] * D0 / 2.0 * grav_fac(a, i, 0, 0, 1, 0);
    double vm0 = a.vm[i];
    double vs0 = a.vs[i];
    double b0_vm = -pos_part(vm0) / dzi[0];
    double b0_vm_B = -neg_part(vm0) / dzi[0];
    double b0_vs = -pos_part(vs0) / dzi[0];
    double b0_vs_B = -neg_part(vs0) / dzi[0];
    double bA = (1.0 - use_vm) * g0 + use_vm * b0_vm + use_set * b0_vs;
    double bB = (1.0 - use_vm) * g0 + use_vm * b0_vm_B + use_set * b0_vs_B;
    A = -1.0 / dzi[0] * (D0 / dzi[0]) * (ysp + ys0) / 2.0 / ys0 + bA;
    Bc = 1.0 / dzi[0] * (D0 / dzi[0]) * (ysp + ys0) / 2.0 / ysp + bB;
    C = 0.0;
  } else if (j == nz - 1) {
    int t = nz - 2;
    double Dt = a.Dzz[(int64_t)t * ni + i];
    double gt = -1.0 / dzi[t] * Dt / 2.0 * grav_fac(a, i, t, nz - 1, nz - 1, nz - 2);
    double vmt = a.vm[(int64_t)(nz - 1) * ni + i];
    double vst = a.vs[(int64_t)t * ni + i];
    double bt_vm = neg_part(vmt) / dzi[t];
    double bt_vm_C = pos_part(vmt) / dzi[t];
    double bt_vs = neg_part(vst) / dzi[t];
    double bt_vs_C = pos_part(vst) / dzi[t];
    double bA = (1.0 - use_vm) * gt + use_vm * bt_vm + use_set * bt_vs;
    double bC = (1.0 - use_vm) * gt + use_vm * bt_vm_C + use_set * bt_vs_C;
    A = -1.0 / dzi[t] * (Dt / dzi[t]) * (ys0 + ysm) / 2.0 / ys0 + bA;
    C = 1.0 / dzi[t] * (Dt / dzi[t]) * (ys0 + ysm) / 2.0 / ysm + bC;
    Bc = 0.0;
  } else {
    double dz_ave = 0.5 * (dzi[j - 1] + dzi[j]);
    double Dj = a.Dzz[(int64_t)j * ni + i];
    double Dm = a.Dzz[(int64_t)(j - 1) * ni + i];
    double gj = grav_fac(a, i, j, j, j + 1, j);
    double gjm = grav_fac(a, i, j - 1, j, j, j - 1);
    double gjpb = grav_fac(a, i, j, j + 1, j + 1, j);
    double gjmc = grav_fac(a, i, j - 1, j - 1, j, j - 1);
    double inv2 = 1.0 / (2.0 * dz_ave);
    double Ag = inv2 * (Dj * gj - Dm * gjm);
    double Bg = inv2 * Dj * gjpb;
    double Cg = -inv2 * Dm * gjmc;
    double vmj = a.vm[(int64_t)j * ni + i], vmm = a.vm[(int64_t)(j - 1) * ni + i];
    double vsj = a.vs[(int64_t)j * ni + i], vsm = a.vs[(int64_t)(j - 1) * ni + i];
    double Avm = -(pos_part(vmj) - neg_part(vmm)) / dz_ave;
    double Bvm = -neg_part(vmj) / dz_ave;
    double Cvm = pos_part(vmm) / dz_ave;
    double Avs = -(pos_part(vsj) - neg_part(vsm)) / dz_ave;
    double Bvs = -neg_part(vsj) / dz_ave;
    double Cvs = pos_part(vsm) / dz_ave;
    double Ax = (1.0 - use_vm) * Ag + use_vm * Avm + use_set * Avs;
    double Bx = (1.0 - use_vm) * Bg + use_vm * Bvm + use_set * Bvs;
    double Cx = (1.0 - use_vm) * Cg + use_vm * Cvm + use_set * Cvs;
    A = -1.0 / dz_ave * (Dj / dzi[j] * (ysp + ys0) / 2.0 + Dm / dzi[j - 1] * (ys0 + ysm) / 2.0) / ys0;
    A = A + Ax;
    Bc = 1.0 / dz_ave * Dj / dzi[j] * (ysp + ys0) / 2.0 / ysp;
    Bc = Bc + Bx;
    C = 1.0 / dz_ave * Dm / dzi[j - 1] * (ys0 + ysm) / 2.0 / ysm;
    C = C + Cx;
  }
}

}  // namespace vb
