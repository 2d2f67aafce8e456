// Photochemistry kernels (reference photo.py):
//   tau_kernel   optical depth, a top-down running sum per wavelength bin
//                (photo.py:84-123);
//   flux_kernel  two-stream Eddington flux: the down and the up recursions in
//                z run in one thread per bin, all bins in parallel
//                (photo.py:126-245);
//   j_kernel     J-rates of a tile of layers and every branch, warp per
//                branch, reductions over bins with the two-resolution
//                trapezoid correction, fused with the write of the photolysis
//                rows of k (photo.py:309-351, 455-478).
// Each kernel takes an optional per-atmosphere mask `due` (atmospheres with
// due[b] == 0 are left alone: the photo branch of the adaptive loop runs only
// where its cadence says so, outer_loop.py:716-724), and the flux kernel an
// optional per-atmosphere accumulator of the actinic-flux change
// (outer_loop.py:327-336), which the tau kernel of the same update zeroes.
// Compiled with --fmad=false: products and sums round as the reference's
// element-wise expressions do.
#include <cuda_runtime.h>

#include "vb_common.cuh"
#include "vb_launch.cuh"

namespace vb {

constexpr int PHOTO_THREADS = 128;
// achg points at VbConvState::aflux_change of atmosphere 0; the records are
// VbConvState-sized apart
constexpr int64_t ACHG_STRIDE = sizeof(VbConvState) / sizeof(double);
static_assert(sizeof(VbConvState) % sizeof(double) == 0, "VbConvState size");

__global__ void __launch_bounds__(PHOTO_THREADS)
tau_kernel(int nz, int ni, VbPhoto P, const double* __restrict__ y, const double* __restrict__ dz,
           double* __restrict__ tau, const int32_t* __restrict__ due, double* __restrict__ achg) {
  const int b = blockIdx.y;
  const int bin = blockIdx.x * blockDim.x + threadIdx.x;
  if (due && due[b] == 0) return;
  if (achg && bin == 0) achg[(int64_t)b * ACHG_STRIDE] = 0.0;
  if (bin >= P.nbin) return;
  const int nbin = P.nbin;
  const double* yb = y + (int64_t)b * nz * ni;
  const double* dzb = dz + (int64_t)b * nz;
  const double* xT = P.absp_T_cross + (int64_t)b * P.T_stride;
  double* tb = tau + (int64_t)b * (nz + 1) * nbin;
  tb[(int64_t)nz * nbin + bin] = 0.0;
  double acc = 0.0;
  for (int j = nz - 1; j >= 0; --j) {
    const double* yj = yb + (int64_t)j * ni;
    double a = 0.0;
    if (P.n_abs > 0) {
      double s = 0.0;
      for (int k = 0; k < P.n_abs; ++k) s = s + yj[P.absp_idx[k]] * P.absp_cross[(int64_t)k * nbin + bin];
      a = s * dzb[j];
    }
    if (P.n_abs_T > 0) {
      double s = 0.0;
      for (int k = 0; k < P.n_abs_T; ++k)
        s = s + yj[P.absp_T_idx[k]] * xT[((int64_t)k * nz + j) * nbin + bin];
      a = a + s * dzb[j];
    }
    if (P.n_scat > 0) {
      double s = 0.0;
      for (int k = 0; k < P.n_scat; ++k) s = s + yj[P.scat_idx[k]] * P.scat_cross[(int64_t)k * nbin + bin];
      a = a + s * dzb[j];
    }
    acc = (j == nz - 1) ? a : acc + a;
    tb[(int64_t)j * nbin + bin] = acc;
  }
}

struct TwoStream {
  double chi, xi, phi, gp, gm;
};

// Single-scattering albedo of one layer and bin (photo.py:150-170): the
// ymix-weighted absorption (T-independent and T-dependent cross sections)
// and scattering sums, w0 = scat / (abs + scat), NaN -> 0, at most 1 - 1e-8.
__device__ inline double albedo(const VbPhoto& P, const double* __restrict__ xT, int nz, const double* ymix_j, int j,
                                int bin) {
  const int nbin = P.nbin;
  double tot_abs = 0.0, tot_scat = 0.0;
  if (P.n_abs > 0) {
    double s = 0.0;
    for (int k = 0; k < P.n_abs; ++k) s = s + ymix_j[P.absp_idx[k]] * P.absp_cross[(int64_t)k * nbin + bin];
    tot_abs = s;
  }
  if (P.n_abs_T > 0) {
    double s = 0.0;
    for (int k = 0; k < P.n_abs_T; ++k)
      s = s + ymix_j[P.absp_T_idx[k]] * xT[((int64_t)k * nz + j) * nbin + bin];
    tot_abs = tot_abs + s;
  }
  if (P.n_scat > 0) {
    double s = 0.0;
    for (int k = 0; k < P.n_scat; ++k) s = s + ymix_j[P.scat_idx[k]] * P.scat_cross[(int64_t)k * nbin + bin];
    tot_scat = s;
  }
  double w0 = tot_scat / fmax(tot_abs + tot_scat, 1e-300);
  if (isnan(w0)) w0 = 0.0;
  return fmin(w0, 1.0 - 1e-8);
}

// Two-stream coefficients of one layer from its albedo (photo.py:171-203).
__device__ inline TwoStream two_stream(const VbPhoto& P, double w0, double dtau) {
  const double mu_ang = -1.0 * P.mu_zenith;
  const double edd = P.edd, ag0 = P.ag0;
  double tran, zp, zm, ll, gp, gm;
  if (ag0 == 0.0) {
    const double sq = sqrt(1.0 - w0);
    tran = exp(-1.0 / edd * sq * dtau);
    zp = 0.5 * (1.0 + sq);
    zm = 0.5 * (1.0 - sq);
    ll = -1.0 * w0 / (1.0 / (mu_ang * mu_ang) - 1.0 / (edd * edd) * (1.0 - w0));
    gp = 0.5 * (ll * (1.0 / edd + 1.0 / mu_ang));
    gm = 0.5 * (ll * (1.0 / edd - 1.0 / mu_ang));
  } else {
    const double wa = 1.0 - w0 * ag0;
    tran = exp(-1.0 / edd * sqrt(wa * (1.0 - w0)) * dtau);
    const double rt = sqrt((1.0 - w0) / wa);
    zp = 0.5 * (1.0 + rt);
    zm = 0.5 * (1.0 - rt);
    ll = ((1.0 - w0) * wa - 1.0) / (1.0 / (mu_ang * mu_ang) - 1.0 / (edd * edd) * (1.0 - w0) * wa);
    gp = 0.5 * (ll * (1.0 / edd + 1.0 / (mu_ang * wa)) + w0 * ag0 * mu_ang / wa);
    gm = 0.5 * (ll * (1.0 / edd - 1.0 / (mu_ang * wa)) - w0 * ag0 * mu_ang / wa);
  }
  TwoStream c;
  c.chi = zm * zm * (tran * tran) - zp * zp;
  c.xi = zp * zm * (1.0 - tran * tran);
  c.phi = (zm * zm - zp * zp) * tran;
  c.gp = gp;
  c.gm = gm;
  return c;
}

__global__ void __launch_bounds__(PHOTO_THREADS)
flux_kernel(int nz, int ni, VbPhoto P, const double* __restrict__ tau, const double* __restrict__ ymix,
            const double* du_prev, double* __restrict__ aflux, double* __restrict__ sflux,
            double* __restrict__ dd, double* du, const int32_t* __restrict__ due, double flux_atol,
            double* __restrict__ achg) {
  // du_prev and du may be one buffer: each thread reads its bin of du_prev in
  // the down recursion before the up recursion overwrites it.
  const int b = blockIdx.y;
  const int bin = blockIdx.x * blockDim.x + threadIdx.x;
  if (due && due[b] == 0) return;
  if (bin >= P.nbin) return;
  const int nbin = P.nbin;
  const int64_t zb = (int64_t)b * (nz + 1) * nbin;
  const double* tb = tau + zb;
  const double* ym = ymix + (int64_t)b * nz * ni;
  const double* xT = P.absp_T_cross + (int64_t)b * P.T_stride;
  const double* up = du_prev + zb;
  double* sb = sflux + zb;
  double* ddb = dd + zb;
  double* dub = du + zb;
  double* ab = aflux + (int64_t)b * nz * nbin;
  const double mu_ang = -1.0 * P.mu_zenith;
  const double top = P.sflux_top[bin];
  // albedo of every layer, parked in the sflux rows until the up recursion
  // hands each row its direct beam (the sums over absorbers run once per
  // layer instead of once per recursion)
  for (int j = 0; j < nz; ++j) sb[(int64_t)j * nbin + bin] = albedo(P, xT, nz, ym + (int64_t)j * ni, j, bin);
  // down recursion (photo.py:208-223), dflux_u of the previous call; the
  // direct beam top * exp(tau / mu) (photo.py:173-174) level by level
  double d_next = 0.0;
  ddb[(int64_t)nz * nbin + bin] = 0.0;
  double s_hi = top * exp(tb[(int64_t)nz * nbin + bin] / mu_ang);
  for (int j = nz - 1; j >= 0; --j) {
    const double t0 = tb[(int64_t)j * nbin + bin], t1 = tb[(int64_t)(j + 1) * nbin + bin];
    const double s_lo = top * exp(t0 / mu_ang);
    TwoStream c = two_stream(P, sb[(int64_t)j * nbin + bin], t0 - t1);
    const double dir0 = s_lo * (-mu_ang);
    const double dir1 = s_hi * (-mu_ang);
    const double i_d = c.phi * c.gm * dir1 - (c.chi * c.gm + c.xi * c.gp) * dir0;
    const double v = (1.0 / c.chi) * (c.phi * d_next - c.xi * up[(int64_t)j * nbin + bin] + i_d / mu_ang);
    ddb[(int64_t)j * nbin + bin] = v;
    d_next = v;
    s_hi = s_lo;
  }
  // up recursion (photo.py:225-236) and the actinic flux (photo.py:238-244)
  double u_prev = 0.0;
  dub[bin] = 0.0;
  const double conv = P.hc / P.bins[bin];
  double change = 0.0;  // largest relative aflux change of this bin (entries above flux_atol)
  double s_lo = top * exp(tb[bin] / mu_ang);
  for (int j = 1; j <= nz; ++j) {
    const double t0 = tb[(int64_t)(j - 1) * nbin + bin], t1 = tb[(int64_t)j * nbin + bin];
    const double s_up = top * exp(t1 / mu_ang);
    TwoStream c = two_stream(P, sb[(int64_t)(j - 1) * nbin + bin], t0 - t1);
    const double dir0 = s_lo * (-mu_ang);
    const double dir1 = s_up * (-mu_ang);
    const double i_u = c.phi * c.gp * dir0 - (c.xi * c.gm + c.chi * c.gp) * dir1;
    const double v = (1.0 / c.chi) * (c.phi * u_prev - c.xi * ddb[(int64_t)j * nbin + bin] + i_u / mu_ang);
    dub[(int64_t)j * nbin + bin] = v;
    const double ave = 0.5 * (s_lo + s_up);
    const double tot = ave + 0.5 * (u_prev + v + ddb[(int64_t)j * nbin + bin] + ddb[(int64_t)(j - 1) * nbin + bin]) / P.edd;
    const double an = tot / conv;
    if (achg && an > flux_atol) {
      const double r = fabs(an - ab[(int64_t)(j - 1) * nbin + bin]) / fmax(fabs(an), 1e-300);
      change = (r > change || r != r) ? r : change;
    }
    ab[(int64_t)(j - 1) * nbin + bin] = an;
    sb[(int64_t)(j - 1) * nbin + bin] = s_lo;   // level j-1's albedo is spent: store its direct beam
    u_prev = v;
    s_lo = s_up;
  }
  sb[(int64_t)nz * nbin + bin] = s_lo;
  // the ratios are >= 0 or NaN, so their bit patterns order as their values
  // do and a NaN wins the maximum, as it does in the reference's max
  if (achg && change != 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(achg + (int64_t)b * ACHG_STRIDE),
              static_cast<unsigned long long>(__double_as_longlong(change)));
}

// J-rates of a tile of JT layers of one atmosphere, all branches: the
// actinic-flux rows of the tile are staged once in shared memory, each warp
// takes every (JW)-th branch, and a branch's cross-section row (shared by
// all layers, unless the branch is temperature dependent) is read once per
// tile (a small batch splits the branches over gridDim.z block groups);
// lanes hold the partial sums of the tile's layers, split at din12
// for the two-resolution trapezoid (photo.py:316-349), then the k row
// (photo.py:465-478).
constexpr int J_THREADS = 256;
constexpr int JW = J_THREADS / 32;
constexpr int JT = 4;

__global__ void __launch_bounds__(J_THREADS)
j_kernel(int nz, int nr, int lt, VbPhoto P, const double* __restrict__ aflux, double* __restrict__ J_br,
         double* __restrict__ J_br_T, double* __restrict__ k, const int32_t* __restrict__ due) {
  extern __shared__ double fs[];   // [lt][nbin]
  const int b = blockIdx.y, j0 = blockIdx.x * lt;
  if (due && due[b] == 0) return;
  const int nbin = P.nbin, d12 = P.din12;
  const int nl = min(lt, nz - j0);
  const double* fb = aflux + ((int64_t)b * nz + j0) * nbin;
  for (int e = threadIdx.x; e < nl * nbin; e += J_THREADS) fs[e] = fb[e];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nb = P.n_br + P.n_br_T;
  for (int br = blockIdx.z * JW + warp; br < nb; br += JW * gridDim.z) {
    const bool is_T = br >= P.n_br;
    const int brl = is_T ? br - P.n_br : br;
    const double* c0 = is_T ? P.cross_J_T + (int64_t)b * P.T_stride_J + ((int64_t)brl * nz + j0) * nbin
                            : P.cross_J + (int64_t)brl * nbin;
    const int64_t cstep = is_T ? nbin : 0;   // next layer's row (T-dependent tables only)
    double s1[JT], s2[JT];
#pragma unroll
    for (int l = 0; l < JT; ++l) s1[l] = s2[l] = 0.0;
    for (int q = lane; q < d12; q += 32) {
#pragma unroll
      for (int l = 0; l < JT; ++l)
        if (l < nl) s1[l] = s1[l] + fs[l * nbin + q] * c0[l * cstep + q];
    }
    for (int q = d12 + lane; q < nbin; q += 32) {
#pragma unroll
      for (int l = 0; l < JT; ++l)
        if (l < nl) s2[l] = s2[l] + fs[l * nbin + q] * c0[l * cstep + q];
    }
#pragma unroll
    for (int l = 0; l < JT; ++l) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        s1[l] = s1[l] + __shfl_xor_sync(0xffffffffu, s1[l], off);
        s2[l] = s2[l] + __shfl_xor_sync(0xffffffffu, s2[l], off);
      }
    }
    if (lane < nl) {
      const int l = lane, j = j0 + l;
      double a1 = 0.0, a2 = 0.0;
#pragma unroll
      for (int t = 0; t < JT; ++t)
        if (t == l) { a1 = s1[t]; a2 = s2[t]; }
      const double* f = fs + l * nbin;
      const double* c = c0 + l * cstep;
      double J = 0.0;
      if (d12 > 0) {
        double J1 = a1 * P.dbin1;
        J1 = J1 - 0.5 * (f[0] * c[0] + f[d12 - 1] * c[d12 - 1]) * P.dbin1;
        J = J1;
      }
      if (d12 < nbin) {
        double J2 = a2 * P.dbin2;
        J2 = J2 - 0.5 * (f[d12] * c[d12] + f[nbin - 1] * c[nbin - 1]) * P.dbin2;
        J = (d12 > 0) ? J + J2 : J2;
      }
      if (is_T) {
        if (J_br_T) J_br_T[((int64_t)b * P.n_br_T + brl) * nz + j] = J;
      } else {
        if (J_br) J_br[((int64_t)b * P.n_br + brl) * nz + j] = J;
      }
      if (k) {
        const int32_t* ridx = is_T ? P.br_T_re_idx : P.br_re_idx;
        const uint8_t* act = is_T ? P.br_T_active : P.br_active;
        if (ridx && act && act[brl]) k[((int64_t)b * (nr + 1) + ridx[brl]) * nz + j] = J * P.f_diurnal;
      }
    }
  }
}

cudaError_t launch_photo_tau(int batch, int nz, int ni, const VbPhoto& P, const double* y, const double* dz,
                             double* tau, const int32_t* due, double* achg, cudaStream_t st) {
  dim3 grid((P.nbin + PHOTO_THREADS - 1) / PHOTO_THREADS, batch);
  tau_kernel<<<grid, PHOTO_THREADS, 0, st>>>(nz, ni, P, y, dz, tau, due, achg);
  return cudaGetLastError();
}

cudaError_t launch_photo_flux(int batch, int nz, int ni, const VbPhoto& P, const double* tau, const double* ymix,
                              const double* du_prev, double* aflux, double* sflux, double* dd, double* du,
                              const int32_t* due, double flux_atol, double* achg, cudaStream_t st) {
  dim3 grid((P.nbin + PHOTO_THREADS - 1) / PHOTO_THREADS, batch);
  flux_kernel<<<grid, PHOTO_THREADS, 0, st>>>(nz, ni, P, tau, ymix, du_prev, aflux, sflux, dd, du, due, flux_atol,
                                              achg);
  return cudaGetLastError();
}

cudaError_t launch_photo_j(int batch, int nz, int nr, const VbPhoto& P, const double* aflux, double* J_br,
                           double* J_br_T, double* k, const int32_t* due, cudaStream_t st) {
  if (P.n_br + P.n_br_T == 0) return cudaSuccess;
  // layers per block: JT when the batch fills the GPU with tiles, else one
  // layer per block (more blocks for a small batch); fewer when the flux rows
  // would not fit 200 KB of shared memory
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int lt = ((int64_t)batch * ((nz + JT - 1) / JT) >= 2 * (int64_t)sms) ? JT : 1;
  while (lt > 1 && (size_t)lt * P.nbin * sizeof(double) > 200 * 1024) --lt;
  if ((size_t)lt * P.nbin * sizeof(double) > 200 * 1024) return cudaErrorInvalidValue;
  const size_t smem = (size_t)lt * P.nbin * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(j_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  // a small batch also spreads its branches over blocks (gridDim.z groups of JW)
  const int groups = lt == 1 ? (P.n_br + P.n_br_T + JW - 1) / JW : 1;
  dim3 grid((nz + lt - 1) / lt, batch, groups);
  j_kernel<<<grid, J_THREADS, smem, st>>>(nz, nr, lt, P, aflux, J_br, J_br_T, k, due);
  return cudaGetLastError();
}

}  // namespace vb
