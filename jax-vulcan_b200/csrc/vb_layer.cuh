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

// Number types of the stencil formulas: double (the forward kernels) or
// Dual (value + one derivative, for the adjoint's leaf cotangents).
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)};
}
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b) { return {a / b.v, -a * b.d / (b.v * b.v)}; }
__device__ __forceinline__ double value_of(double x) { return x; }
__device__ __forceinline__ double value_of(Dual x) { return x.v; }
template <typename T> __device__ __forceinline__ T pos_part_t(T v) { return (value_of(v) > 0.0 ? 1.0 : 0.0) * v; }
template <typename T> __device__ __forceinline__ T neg_part_t(T v) { return (value_of(v) < 0.0 ? 1.0 : 0.0) * v; }

// Plain reads of an atmosphere (the forward kernels).
struct AtmPtrAcc {
  const AtmRef& a;
  int ni;
  __device__ double Kzz(int m) const { return a.Kzz[m]; }
  __device__ double dzi(int m) const { return a.dzi[m]; }
  __device__ double vz(int m) const { return a.vz[m]; }
  __device__ double Hpi(int m) const { return a.Hpi[m]; }
  __device__ double Ti(int m) const { return a.Ti[m]; }
  __device__ double Tco(int m) const { return a.Tco[m]; }
  __device__ double g(int m) const { return a.g[m]; }
  __device__ double Dzz(int m, int i) const { return a.Dzz[(int64_t)m * ni + i]; }
  __device__ double vm(int m, int i) const { return a.vm[(int64_t)m * ni + i]; }
  __device__ double vs(int m, int i) const { return a.vs[(int64_t)m * ni + i]; }
  __device__ double ms(int i) const { return a.ms[i]; }
  __device__ double alpha(int i) const { return a.alpha[i]; }
};

// The atmosphere fields stencil row j reads, staged before any arithmetic:
// the per-layer fields of layers j-1, j, j+1 in shared memory (lay[f][s],
// f = Kzz dzi vz Hpi Ti Tco g, s = layer - (j-1); stage_row_layers) and one
// species' fields of layers j-1, j in registers. eddy_row_t and mol_row_t
// read only those indices for row j (boundary rows included), so this
// accessor returns the values AtmPtrAcc would, without their global-load
// latency between the divisions.
struct RowAcc {
  const double* lay;
  int j0;                                   // j - 1
  double Dm, Dj, vmm, vmj, vsm, vsj, ms_, alpha_;
  int base, S;                              // lay[f * S + m - base]: the staged layers base.. of field f
  __device__ int at(int f, int m) const { return f * S + m - base; }
  __device__ double Kzz(int m) const { return lay[at(0, m)]; }
  __device__ double dzi(int m) const { return lay[at(1, m)]; }
  __device__ double vz(int m) const { return lay[at(2, m)]; }
  __device__ double Hpi(int m) const { return lay[at(3, m)]; }
  __device__ double Ti(int m) const { return lay[at(4, m)]; }
  __device__ double Tco(int m) const { return lay[at(5, m)]; }
  __device__ double g(int m) const { return lay[at(6, m)]; }
  __device__ double Dzz(int m, int) const { return m == j0 ? Dm : Dj; }
  __device__ double vm(int m, int) const { return m == j0 ? vmm : vmj; }
  __device__ double vs(int m, int) const { return m == j0 ? vsm : vsj; }
  __device__ double ms(int) const { return ms_; }
  __device__ double alpha(int) const { return alpha_; }
};

// Fills lay[7][3] for row j (threads 0..20; layers outside [0, nz) read 0).
__device__ inline void stage_row_layers(const AtmRef& a, int nz, int j, double* lay) {
  if (threadIdx.x < 21) {
    const int f = threadIdx.x / 3, m = j - 1 + (int)threadIdx.x % 3;
    const double* src = f == 0 ? a.Kzz : f == 1 ? a.dzi : f == 2 ? a.vz : f == 3 ? a.Hpi : f == 4 ? a.Ti
                      : f == 5 ? a.Tco : a.g;
    lay[threadIdx.x] = (m >= 0 && m < nz) ? src[m] : 0.0;
  }
}

// The staged per-layer fields only (lay[f][3] of row j; the eddy terms).
__device__ inline RowAcc layer_acc(const double* lay, int j) {
  RowAcc R{};
  R.lay = lay;
  R.j0 = j - 1;
  R.base = j - 1;
  R.S = 3;
  return R;
}

// A species' fields of layers j-1 and j, loaded together (lay: per-layer
// fields staged with f-stride S from layer base; a row's own stage: j-1, 3).
__device__ inline RowAcc row_acc(const AtmRef& a, const double* lay, int ni, int j, int i, int base, int S) {
  RowAcc R;
  R.lay = lay;
  R.j0 = j - 1;
  R.base = base;
  R.S = S;
  const int64_t cj = (int64_t)j * ni + i, cm = cj - ni;
  R.Dj = a.Dzz[cj];
  R.vmj = a.vm[cj];
  R.vsj = a.vs[cj];
  R.Dm = j > 0 ? a.Dzz[cm] : 0.0;
  R.vmm = j > 0 ? a.vm[cm] : 0.0;
  R.vsm = j > 0 ? a.vs[cm] : 0.0;
  R.ms_ = a.ms[i];
  R.alpha_ = a.alpha[i];
  return R;
}

// Eddy coefficients of stencil row j (reference jax_step.py:167-193).
template <typename T, typename Acc>
__device__ inline void eddy_row_t(const Acc& a, int nz, int j, double ysm, double ys0, double ysp, T& A, T& Bc,
                                  T& C) {
  if (j == 0) {
    A = -1.0 / a.dzi(0) * (a.Kzz(0) / a.dzi(0)) * (ysp + ys0) / 2.0 / ys0;
    A = A - pos_part_t(a.vz(0)) / a.dzi(0);
    Bc = 1.0 / a.dzi(0) * (a.Kzz(0) / a.dzi(0)) * (ysp + ys0) / 2.0 / ysp;
    Bc = Bc - neg_part_t(a.vz(0)) / a.dzi(0);
    C = T{};
  } else if (j == nz - 1) {
    int t = nz - 2;
    A = -1.0 / a.dzi(t) * (a.Kzz(t) / a.dzi(t)) * (ys0 + ysm) / 2.0 / ys0;
    A = A + neg_part_t(a.vz(t)) / a.dzi(t);
    C = 1.0 / a.dzi(t) * (a.Kzz(t) / a.dzi(t)) * (ys0 + ysm) / 2.0 / ysm;
    C = C + pos_part_t(a.vz(t)) / a.dzi(t);
    Bc = T{};
  } else {
    const auto dz_ave = 0.5 * (a.dzi(j - 1) + a.dzi(j));
    A = -1.0 / dz_ave *
        (a.Kzz(j) / a.dzi(j) * (ysp + ys0) / 2.0 + a.Kzz(j - 1) / a.dzi(j - 1) * (ys0 + ysm) / 2.0) / ys0;
    Bc = 1.0 / dz_ave * a.Kzz(j) / a.dzi(j) * (ysp + ys0) / 2.0 / ysp;
    C = 1.0 / dz_ave * a.Kzz(j - 1) / a.dzi(j - 1) * (ys0 + ysm) / 2.0 / ysm;
    A = A - (pos_part_t(a.vz(j)) - neg_part_t(a.vz(j - 1))) / dz_ave;
    Bc = Bc - neg_part_t(a.vz(j)) / dz_ave;
    C = C + pos_part_t(a.vz(j - 1)) / dz_ave;
  }
}

__device__ inline void eddy_row(const AtmRef& a, int nz, int j, double ysm, double ys0, double ysp,
                                double& A, double& Bc, double& C) {
  eddy_row_t<double>(AtmPtrAcc{a, 0}, nz, j, ysm, ys0, ysp, A, Bc, C);
}

// Gravity/thermal-diffusion factor of compute_diff_grav (jax_step.py:80-87):
// -1/Hpi[h] + ms*g[gi]/(Navo*kb*Ti[h]) + alpha/Ti[h]*(Tco[t1]-Tco[t0])/dzi[h].
template <typename T, typename Acc>
__device__ __forceinline__ T grav_fac_t(const Acc& a, int i, int h, int gi, int t1, int t0) {
  return -1.0 / a.Hpi(h) + a.ms(i) * a.g(gi) / (NAVO * KB * a.Ti(h)) +
         a.alpha(i) / a.Ti(h) * (a.Tco(t1) - a.Tco(t0)) / a.dzi(h);
}

// Molecular-diffusion coefficients of species i on stencil row j, including the
// y-independent gravity / vm / settling pieces (jax_step.py:67-147, 195-218).
template <typename T, typename Acc>
__device__ inline void mol_row_t(const Acc& a, int nz, int j, int i, double ysm, double ys0, double ysp,
                                 double use_vm, double use_set, T& A, T& Bc, T& C) {
  if (j == 0) {
    const T D0 = a.Dzz(0, i);
    const T g0 = 1.0 / a.dzi(0) * D0 / 2.0 * grav_fac_t<T>(a, i, 0, 0, 1, 0);
    const T vm0 = a.vm(0, i);
    const T vs0 = a.vs(0, i);
    const T b0_vm = -pos_part_t(vm0) / a.dzi(0);
    const T b0_vm_B = -neg_part_t(vm0) / a.dzi(0);
    const T b0_vs = -pos_part_t(vs0) / a.dzi(0);
    const T b0_vs_B = -neg_part_t(vs0) / a.dzi(0);
    const T bA = (1.0 - use_vm) * g0 + use_vm * b0_vm + use_set * b0_vs;
    const T bB = (1.0 - use_vm) * g0 + use_vm * b0_vm_B + use_set * b0_vs_B;
    A = -1.0 / a.dzi(0) * (D0 / a.dzi(0)) * (ysp + ys0) / 2.0 / ys0 + bA;
    Bc = 1.0 / a.dzi(0) * (D0 / a.dzi(0)) * (ysp + ys0) / 2.0 / ysp + bB;
    C = T{};
  } else if (j == nz - 1) {
    const int t = nz - 2;
    const T Dt = a.Dzz(t, i);
    const T gt = -1.0 / a.dzi(t) * Dt / 2.0 * grav_fac_t<T>(a, i, t, nz - 1, nz - 1, nz - 2);
    const T vmt = a.vm(nz - 1, i);
    const T vst = a.vs(t, i);
    const T bt_vm = neg_part_t(vmt) / a.dzi(t);
    const T bt_vm_C = pos_part_t(vmt) / a.dzi(t);
    const T bt_vs = neg_part_t(vst) / a.dzi(t);
    const T bt_vs_C = pos_part_t(vst) / a.dzi(t);
    const T bA = (1.0 - use_vm) * gt + use_vm * bt_vm + use_set * bt_vs;
    const T bC = (1.0 - use_vm) * gt + use_vm * bt_vm_C + use_set * bt_vs_C;
    A = -1.0 / a.dzi(t) * (Dt / a.dzi(t)) * (ys0 + ysm) / 2.0 / ys0 + bA;
    C = 1.0 / a.dzi(t) * (Dt / a.dzi(t)) * (ys0 + ysm) / 2.0 / ysm + bC;
    Bc = T{};
  } else {
    const T dz_ave = 0.5 * (a.dzi(j - 1) + a.dzi(j));
    const T Dj = a.Dzz(j, i);
    const T Dm = a.Dzz(j - 1, i);
    const T gj = grav_fac_t<T>(a, i, j, j, j + 1, j);
    const T gjm = grav_fac_t<T>(a, i, j - 1, j, j, j - 1);
    const T gjpb = grav_fac_t<T>(a, i, j, j + 1, j + 1, j);
    const T gjmc = grav_fac_t<T>(a, i, j - 1, j - 1, j, j - 1);
    const T inv2 = 1.0 / (2.0 * dz_ave);
    const T Ag = inv2 * (Dj * gj - Dm * gjm);
    const T Bg = inv2 * Dj * gjpb;
    const T Cg = -inv2 * Dm * gjmc;
    const T vmj = a.vm(j, i), vmm = a.vm(j - 1, i);
    const T vsj = a.vs(j, i), vsm = a.vs(j - 1, i);
    const T Avm = -(pos_part_t(vmj) - neg_part_t(vmm)) / dz_ave;
    const T Bvm = -neg_part_t(vmj) / dz_ave;
    const T Cvm = pos_part_t(vmm) / dz_ave;
    const T Avs = -(pos_part_t(vsj) - neg_part_t(vsm)) / dz_ave;
    const T Bvs = -neg_part_t(vsj) / dz_ave;
    const T Cvs = pos_part_t(vsm) / dz_ave;
    const T Ax = (1.0 - use_vm) * Ag + use_vm * Avm + use_set * Avs;
    const T Bx = (1.0 - use_vm) * Bg + use_vm * Bvm + use_set * Bvs;
    const T Cx = (1.0 - use_vm) * Cg + use_vm * Cvm + use_set * Cvs;
    A = -1.0 / dz_ave * (Dj / a.dzi(j) * (ysp + ys0) / 2.0 + Dm / a.dzi(j - 1) * (ys0 + ysm) / 2.0) / ys0;
    A = A + Ax;
    Bc = 1.0 / dz_ave * Dj / a.dzi(j) * (ysp + ys0) / 2.0 / ysp;
    Bc = Bc + Bx;
    C = 1.0 / dz_ave * Dm / a.dzi(j - 1) * (ys0 + ysm) / 2.0 / ysm;
    C = C + Cx;
  }
}

__device__ inline void mol_row(const AtmRef& a, int nz, int ni, int j, int i, double ysm, double ys0,
                               double ysp, double use_vm, double use_set, double& A, double& Bc,
                               double& C) {
  mol_row_t<double>(AtmPtrAcc{a, ni}, nz, j, i, ysm, ys0, ysp, use_vm, use_set, A, Bc, C);
}

}  // namespace vb
