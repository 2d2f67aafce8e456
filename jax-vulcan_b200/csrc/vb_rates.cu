// Rate constants on the device (reference rates.py:61-208, gibbs.py:41-150).
// One thread per (layer, reaction pair): the forward constant of row i
// (odd), the low-temperature cap, the equilibrium constant from the NASA-9
// g/RT of its species (evaluated in place, no workspace) and the reverse
// constant of row i+1, then the removal mask. The layer index runs along
// threadIdx.x, so the stores of k[B][nr+1][nz] are coalesced.
//
// Templated on the number type: double gives k; Dual (value, d/dT) gives k
// and dk/dT from the same expressions, the value part rounding exactly as the
// double path. Compiled with --fmad=false, and the powers follow NumPy's
// scalar-exponent shortcuts (x**2 -> x*x, x**-1 -> 1/x, x**0.5 -> sqrt,
// x**0 -> 1, x**1 -> x), so products and sums round as the reference's
// element-wise expressions do; exp, log and pow are CUDA's (within a few ulp
// of the host libm).
#include <cuda_runtime.h>

#include "vb_common.cuh"
#include "vb_launch.cuh"
#include "vb_layer.cuh"

namespace vb {

constexpr int RATE_THREADS = 128;
constexpr double K_BOLTZ = 1.38064852e-16;  // erg/K
constexpr double CORR = K_BOLTZ / 1.0e6;     // k_B / P0 of the equilibrium constant

__device__ __forceinline__ double r_exp(double x) { return exp(x); }
__device__ __forceinline__ double r_log(double x) { return log(x); }
__device__ __forceinline__ Dual r_exp(Dual x) {
  const double e = exp(x.v);
  return {e, e * x.d};
}
__device__ __forceinline__ Dual r_log(Dual x) { return {log(x.v), x.d / x.v}; }

// x ** e for a scalar exponent, with NumPy's shortcuts
__device__ __forceinline__ double r_pow(double x, double e) {
  if (e == 2.0) return x * x;
  if (e == 1.0) return x;
  if (e == 0.0) return 1.0;
  if (e == -1.0) return 1.0 / x;
  if (e == 0.5) return sqrt(x);
  return pow(x, e);
}
__device__ __forceinline__ Dual r_pow(Dual x, double e) {
  const double v = r_pow(x.v, e);
  double dv;
  if (e == 0.0) dv = 0.0;
  else if (e == 1.0) dv = 1.0;
  else if (e == 2.0) dv = 2.0 * x.v;
  else dv = e * pow(x.v, e - 1.0);
  return {v, dv * x.d};
}

template <typename N> __device__ __forceinline__ N arrhenius(double a, double n, double E, N T) {
  return a * r_pow(T, n) * r_exp(-E / T);
}

// Troe falloff of OH + CH3 + M -> CH3OH + M (rates.py:41-58)
template <typename N> __device__ N troe_oh_ch3(N T, double M) {
  const N k0 = 1.932e3 * r_pow(T, -9.88) * r_exp(-7544.0 / T) + 5.109e-11 * r_pow(T, -6.25) * r_exp(-1433.0 / T);
  const N kinf = 1.031e-10 * r_pow(T, -0.018) * r_exp(16.74 / T);
  const N Fc = 0.1855 * r_exp(-T / 155.8) + 0.8145 * r_exp(-T / 1675.0) + r_exp(-4531.0 / T);
  const N nn = 0.75 - 1.27 * r_log(Fc);
  const N q = r_log(k0 * M / kinf) / nn;
  const N ff = r_exp(r_log(Fc) / (1.0 + q * q));
  return k0 / (1.0 + k0 * M / kinf) * ff;
}

// g/RT of one species (gibbs.py:47-73): H/RT - S/R of the branch T selects
template <typename N> __device__ N gibbs(const double* __restrict__ c9, N T) {
  const double* a = c9 + (value_of(T) < 1000.0 ? 0 : 10);
  const N lT = r_log(T);
  const N T2 = r_pow(T, 2.0), T3 = r_pow(T, 3.0), T4 = r_pow(T, 4.0);
  const N h = -a[0] / T2 + a[1] * lT / T + a[2] + a[3] * T / 2.0 + a[4] * T2 / 3.0 + a[5] * T3 / 4.0 +
              a[6] * T4 / 5.0 + a[8] / T;
  const N s = -a[0] / T2 / 2.0 - a[1] / T + a[2] * lT + a[3] * T + a[4] * T2 / 2.0 + a[5] * T3 / 3.0 +
              a[6] * T4 / 4.0 + a[9];
  return h - s;
}

__device__ __forceinline__ void store(double* k, double* dk, int64_t at, double v) {
  k[at] = v;
  if (dk) dk[at] = 0.0;
}
__device__ __forceinline__ void store(double* k, double* dk, int64_t at, Dual v) {
  k[at] = v.v;
  dk[at] = v.d;
}

template <typename N>
__global__ void __launch_bounds__(RATE_THREADS)
rates_kernel(int nz, VbRateTables t, const double* __restrict__ Tp, const double* __restrict__ Mp, int flags,
             double* __restrict__ k, double* __restrict__ dk) {
  const int z = blockIdx.x * RATE_THREADS + threadIdx.x;
  const int pair = blockIdx.y, b = blockIdx.z;
  if (z >= nz) return;
  const int i = 2 * pair + 1;
  const int64_t rows = (int64_t)(t.nr + 1) * nz;
  double* kb = k + (int64_t)b * rows;
  double* db = dk ? dk + (int64_t)b * rows : nullptr;
  if (pair == 0) store(kb, db, z, 0.0);   // row 0 is unused
  const double Tv = Tp[(int64_t)b * nz + z];
  const double M = Mp[(int64_t)b * nz + z];
  N T;
  if constexpr (sizeof(N) == sizeof(double)) T = Tv;
  else T = N{Tv, 1.0};
  const int code = t.code[i];
  const double* par = t.par + (int64_t)i * 6;
  N kf = N{};
  switch (code & 3) {
    case VB_RK_ARRHENIUS: kf = arrhenius(par[0], par[1], par[2], T); break;
    case VB_RK_LINDEMANN: {
      const N k0 = arrhenius(par[0], par[1], par[2], T);
      const N kinf = arrhenius(par[3], par[4], par[5], T);
      kf = k0 / (1.0 + k0 * M / kinf);
      break;
    }
    case VB_RK_TROE_OH_CH3: kf = troe_oh_ch3(T, M); break;
    default: break;
  }
  const int cap = (code >> 2) & 3;
  if ((flags & VB_RATES_LOWT_CAPS) && cap) {   // rates.py:141-166
    if (cap == VB_RCAP_CH3 && Tv <= 277.5) {
      const double k0 = 6.0e-29;
      const N kinf = 2.06e-10 * r_pow(T, -0.4);
      kf = k0 / (1.0 + k0 * M / kinf);
    } else if (cap == VB_RCAP_C2H4 && Tv <= 300.0) {
      kf = N{} + 3.7e-30;
    } else if (cap == VB_RCAP_C2H5 && Tv <= 200.0) {
      kf = N{} + 2.49e-27;
    }
  }
  N kr = N{};
  if (code & VB_RC_REVERSE) {
    N K = N{} + 1.0;
    if (code & VB_RC_THERMAL) {   // gibbs.py:104-123
      const int T_ = t.max_terms;
      N rs = N{}, ps = N{};
      double dn_r = 0.0, dn_p = 0.0;
      for (int s = 0; s < T_; ++s) {
        const double st = t.r_st[(int64_t)i * T_ + s];
        dn_r = dn_r + st;
        if (st != 0.0) {
          const int sp = t.r_idx[(int64_t)i * T_ + s];
          rs = rs + st * (sp < t.ni ? gibbs(t.nasa9 + (int64_t)sp * 20, T) : N{});
        }
      }
      for (int s = 0; s < T_; ++s) {
        const double st = t.p_st[(int64_t)i * T_ + s];
        dn_p = dn_p + st;
        if (st != 0.0) {
          const int sp = t.p_idx[(int64_t)i * T_ + s];
          ps = ps + st * (sp < t.ni ? gibbs(t.nasa9 + (int64_t)sp * 20, T) : N{});
        }
      }
      const double dn = dn_r - dn_p;
      K = r_exp(rs - ps);
      if (dn != 0.0) K = K * r_pow(CORR * T, dn);
    }
    if (value_of(K) > 0.0) kr = kf / K;   // gibbs.py:138-143
  }
  const int64_t at = (int64_t)i * nz + z;
  store(kb, db, at, (code & VB_RC_DROP_FWD) ? N{} : kf);
  store(kb, db, at + nz, (code & VB_RC_DROP_REV) ? N{} : kr);
}

cudaError_t launch_rates(int batch, int nz, const VbRateTables& t, const double* T, const double* M, int flags,
                         double* k, double* dkdT, cudaStream_t st) {
  dim3 grid((nz + RATE_THREADS - 1) / RATE_THREADS, t.nr / 2, batch);
  if (dkdT)
    rates_kernel<Dual><<<grid, RATE_THREADS, 0, st>>>(nz, t, T, M, flags, k, dkdT);
  else
    rates_kernel<double><<<grid, RATE_THREADS, 0, st>>>(nz, t, T, M, flags, k, nullptr);
  return cudaGetLastError();
}

}  // namespace vb
