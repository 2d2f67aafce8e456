// Layer-parallel assembly kernels of the Ros2 step: chemistry RHS (mass-action
// rates gathered per species), analytic Jacobian (gathered per destination
// entry), eddy + molecular diffusion and boundary fluxes, fused into
//   * the stage-1 kernel: rhs(y) and the LHS blocks c0*I - J - diag(diff)
//     (reference jax_step.py:263-298, chem.py:83-214), and
//   * the stage-2 kernel: rhs(yk2) - 2/(r dt) k1 (jax_step.py:303-310).
// One CTA per (layer, atmosphere). Compiled with --fmad=false: the gathers sum
// in the segment_sum order of the reference, so the RHS and the Jacobian are
// bit-identical to the reference's.
#include <cuda_runtime.h>

#include <algorithm>

#include "vb_common.cuh"
#include "vb_launch.cuh"
#include "vb_layer.cuh"

namespace vb {

struct LayerSmem {
  double* y3;      // [3][ni+1]: layers j-1, j, j+1 (padding slot = 1.0)
  double* rate;    // [nr+1]
  double* drate;   // [(nr+1)*T]
  double* jac;     // [ni*ni] gathered Jacobian
  double* diff;    // [ni]
  double* diagd;   // [ni]
  double* part;    // [2*ni] loss / production partial sums
  double* scal;    // [8]: ysum(j-1), ysum(j), ysum(j+1)
};

// jac: drate buffer for the Jacobian; jsm: also a shared-memory Jacobian block.
__host__ __device__ inline size_t layer_smem_bytes(int ni, int nr, int T, bool jac, bool jsm = false) {
  size_t d = 3 * (size_t)(ni + 1) + (nr + 1) + (jac ? (size_t)(nr + 1) * T : 0) + (jsm ? (size_t)ni * ni : 0) +
             4 * (size_t)ni + 8;
  return d * sizeof(double);
}

__device__ inline LayerSmem carve(double* s, int ni, int nr, int T, bool jac, bool jsm = false) {
  LayerSmem L;
  L.y3 = s; s += 3 * (ni + 1);
  L.rate = s; s += nr + 1;
  L.drate = s; s += jac ? (nr + 1) * T : 0;
  L.jac = s; s += jsm ? ni * ni : 0;
  L.diff = s; s += ni;
  L.diagd = s; s += ni;
  L.part = s; s += 2 * ni;
  L.scal = s;
  return L;
}

// Rate of one reaction from its reactant values yr[] and stoichiometries
// st[] (padding slots st = 0), and with jac its derivative by each reactant
// slot into d[], in the reference's expression order (chem.py:92-99,
// 156-182). Shared by the per-layer and the layer-vectorized assembly.
template <int TT>
__device__ __forceinline__ double rate_terms(const double (&yr)[TT], const double (&st)[TT], double kr, double M,
                                             bool three, bool jac, double (&d)[TT]) {
  double f[TT];
#pragma unroll
  for (int s = 0; s < TT; ++s) f[s] = st[s] > 0.0 ? pow_st(yr[s], st[s]) : 1.0;
  double prod = f[0];
#pragma unroll
  for (int s = 1; s < TT; ++s) prod = prod * f[s];
  double rt = kr * prod;
  if (three) rt = rt * M;
  if (jac) {
#pragma unroll
    for (int s = 0; s < TT; ++s) {
      double lo = (s == 0) ? 1.0 : f[0];
#pragma unroll
      for (int t = 1; t < TT; ++t) lo = lo * ((t == s) ? 1.0 : f[t]);
      double pm1 = st[s] > 0.0 ? pow_st(yr[s], st[s] - 1.0) : 0.0;
      double dd = st[s] * pm1;
      dd = dd * lo;
      dd = dd * kr;
      if (three) dd = dd * M;
      d[s] = dd;
    }
  }
  return rt;
}

// Rate (and drate) of reaction slot r with TT terms of one layer.
template <int TT>
__device__ inline void rate_slot(const NetDev& net, int r, const double* yrow, double kr, double M, double* rate,
                                 double* drate, bool jac) {
  double yr[TT], st[TT], d[TT];
#pragma unroll
  for (int s = 0; s < TT; ++s) {
    st[s] = net.r_st[r * TT + s];
    yr[s] = yrow[net.r_idx[r * TT + s]];
  }
  rate[r] = rate_terms<TT>(yr, st, kr, M, net.three[r] != 0, jac, d);
  if (jac) {
#pragma unroll
    for (int s = 0; s < TT; ++s) drate[r * TT + s] = d[s];
  }
}

// Rate constants of RU consecutive passes, loaded before any arithmetic so the
// strided L2 loads overlap (L2 only: the column of k would flush the gather
// tables from L1).
template <int TT, int RU>
__device__ inline void rates_t(const NetDev& net, const double* yrow, const double* kcol, int64_t kstride, double M,
                               double* rate, double* drate, bool jac) {
  for (int r0 = threadIdx.x; r0 <= net.nr; r0 += RU * blockDim.x) {
    double kv[RU];
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int r = r0 + u * blockDim.x;
      kv[u] = r <= net.nr ? __ldcg(kcol + (int64_t)r * kstride) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int r = r0 + u * blockDim.x;
      if (r <= net.nr) rate_slot<TT>(net, r, yrow, kv[u], M, rate, drate, jac);
    }
  }
}

// rate[r] = k[r] * prod_s y^st (* M) for every reaction slot of one layer
// (chem.py:92-99); with jac, also drate[r][s] (chem.py:156-182).
__device__ inline void layer_rates(const NetDev& net, const double* yrow, const double* kcol,
                                   int64_t kstride, double M, double* rate, double* drate, bool jac) {
  if (!jac) {   // the right-hand-side kernels run at full occupancy: fewer loads in flight per thread
    switch (net.T) {
      case 1: rates_t<1, 2>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
      case 2: rates_t<2, 2>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
      case 3: rates_t<3, 2>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
      case 4: rates_t<4, 2>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
      case 5: rates_t<5, 2>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
      case 6: rates_t<6, 2>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
      case 7: rates_t<7, 2>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
      default: rates_t<8, 2>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
    }
  }
  switch (net.T) {
    case 1: rates_t<1, 6>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
    case 2: rates_t<2, 6>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
    case 3: rates_t<3, 6>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
    case 4: rates_t<4, 6>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
    case 5: rates_t<5, 4>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
    case 6: rates_t<6, 4>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
    case 7: rates_t<7, 4>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
    default: rates_t<8, 4>(net, yrow, kcol, kstride, M, rate, drate, jac); return;
  }
}

// Loss and production sums of every species, each a sequential gather in
// segment_sum order (one thread per sum): part[2i] = loss_i, part[2i+1] = prod_i.
// The caller synchronises before reading dy_i/dt = part[2i+1] - part[2i].
__device__ inline void species_sums(const NetDev& net, const double* coef, const double* rate, double* part) {
  for (int t = threadIdx.x; t < 2 * net.ni; t += blockDim.x) {
    const uint2 d = net.sum_desc[t];
    double acc = 0.0;
    const int e1 = (int)d.x + 32 * (int)d.y;
#pragma unroll 4
    for (int e = (int)d.x; e < e1; e += 32) {
      const uint32_t x = net.sum_w[e];
      acc = acc + coef[x >> 16] * rate[x & 0xffffu];
    }
    part[t] = acc;
  }
}

// The coefficient table of the gathers into shared memory (coef[MAX_COEF]).
__device__ inline void load_coefs(const NetDev& net, double* coef) {
  for (int c = threadIdx.x; c < net.n_coef; c += blockDim.x) coef[c] = net.coef_tab[c];
}

// Dense Jacobian of one layer (chem.py:183-208), each entry summed in the
// reference's scatter order. Threads take the destinations in rank bands of
// decreasing term count (jac_desc), so the lanes of a warp run loops of
// similar length; the terms of 32 consecutive ranks are interleaved in
// jac_w (term i of a rank at its first word + 32 i), so a warp whose lanes
// hold one such group reads one 128-byte line per term.
// busy: the first threads are also summing species lists in the same phase;
// the rank bands are rotated (by whole warps, keeping the groups aligned) so
// those threads take the lightest ranks of each band.
__device__ inline int warp_rotation(int busy) { return (busy + 31) & ~31; }

template <typename Store>
__device__ inline void layer_jacobian_each(const NetDev& net, const double* coef, const double* drate, Store store,
                                           int busy = 0) {
  const int nd = net.ni * net.ni;
  const int stride = blockDim.x;
  int q = ((int)threadIdx.x - warp_rotation(busy) % stride + stride) % stride;
  uint2 dn = q < nd ? net.jac_desc[q] : make_uint2(0u, 0u);
  for (; q < nd; q += stride) {
    const uint2 dc = dn;
    if (q + stride < nd) dn = net.jac_desc[q + stride];   // the next destination's descriptor, one ahead
    const int e0 = (int)dc.x, e1 = e0 + 32 * (int)(dc.y & 0xffffu);
    double J = 0.0;
#pragma unroll 4
    for (int e = e0; e < e1; e += 32) {
      const uint32_t x = net.jac_w[e];
      J = J + coef[x >> 16] * drate[x & 0xffffu];
    }
    store((int)((dc.y >> 16) & 0xffu), (int)(dc.y >> 24), J);
  }
}

__device__ inline void layer_jacobian(const NetDev& net, const double* coef, const double* drate, double* jac) {
  const int ni = net.ni;
  layer_jacobian_each(net, coef, drate, [&](int row, int col, double J) { jac[row * ni + col] = J; });
}

// Loads state rows j-1..j+1 (stage 2: yk2 = y + k1/r) and their gas sums.
template <bool STAGE_GAS = false>
__device__ inline void load_rows(const double* y, const double* k1, const double* gas, int nz, int ni,
                                 int j, double rinv_r, bool stage2, LayerSmem& L) {
  for (int t = threadIdx.x; t < 3 * (ni + 1); t += blockDim.x) {
    int w = t / (ni + 1), i = t % (ni + 1);
    int jj = j - 1 + w;
    double v = 1.0;
    if (i < ni) {
      if (jj >= 0 && jj < nz) {
        v = y[(int64_t)jj * ni + i];
        if (stage2) v = v + k1[(int64_t)jj * ni + i] / rinv_r;
      } else {
        v = 0.0;
      }
    }
    L.y3[t] = v;
  }
  // STAGE_GAS: the gas mask staged in diagd (free until the diffusion writes
  // it), so the three sums below read shared memory
  if (STAGE_GAS)
    for (int i = threadIdx.x; i < ni; i += blockDim.x) L.diagd[i] = gas[i];
  __syncthreads();
  if (threadIdx.x < 3) {
    int w = threadIdx.x;
    int jj = j - 1 + w;
    double s = 0.0;
    if (jj >= 0 && jj < nz) s = pairwise_sum_masked(L.y3 + w * (ni + 1), STAGE_GAS ? L.diagd : gas, ni);
    L.scal[w] = s;
  }
  __syncthreads();
}

// diff[i] (with BC fluxes) and the diagonal diffusion term diag_d[i] of row j;
// also the sup/sub coefficients of row j when requested.
// Diffusion term of species i on row j from its combined coefficients and
// state values y(j), y(j-1), y(j+1): the stencil and the boundary fluxes
// (jax_step.py:223-246, _apply_diffusion_jax).
__device__ inline double diffusion_term(const AtmRef& a, int nz, int j, int i, int flags, double At, double Bt,
                                        double Ct, double y0, double ym, double yp) {
  double d;
  if (j == 0) {
    d = At * y0 + Bt * yp;
  } else if (j == nz - 1) {
    d = At * y0 + Ct * ym;
  } else {
    d = At * y0 + Bt * yp + Ct * ym;
  }
  if (j == nz - 1) {
    d = d + ((flags & VB_USE_TOPFLUX) ? a.top[i] / a.dzi[nz - 2] : 0.0);
  }
  if (j == 0) {
    d = d + ((flags & VB_USE_BOTFLUX) ? (a.bot[i] - y0 * a.vdep[i]) / a.dzi[0] : 0.0);
  }
  return d;
}

// STAGED 2: the row's atmosphere fields are loaded in one round before the
// arithmetic (RowAcc: per-layer fields in shared memory, the species' own in
// registers; faster in the stage-2 kernels, slower in stage 1, where the
// extra live registers spill); 0: read where used. again: a second call in
// the same kernel (waits until the first has read eddy and lay).
template <int STAGED = 0>
__device__ inline void layer_diffusion(const AtmRef& a, int nz, int ni, int j, int flags, LayerSmem& L,
                                       double* sup_out, double* sub_out, bool want_diag, bool again = false) {
  double ysm = L.scal[0], ys0 = L.scal[1], ysp = L.scal[2];
  // the row's per-layer fields staged in one round of loads (the eddy and
  // molecular terms then read them between their divisions from shared
  // memory; each species' own fields are loaded together below)
  __shared__ double eddy[3], lay[21];
  if (again) __syncthreads();   // the previous call has finished reading eddy and lay
  if (STAGED) {
    stage_row_layers(a, nz, j, lay);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double A, B, C;
    if (STAGED)
      eddy_row_t<double>(layer_acc(lay, j), nz, j, ysm, ys0, ysp, A, B, C);
    else
      eddy_row(a, nz, j, ysm, ys0, ysp, A, B, C);
    eddy[0] = A; eddy[1] = B; eddy[2] = C;
  }
  __syncthreads();
  double use_vm = (flags & VB_USE_VM_MOL) ? 1.0 : 0.0;
  double use_set = (flags & VB_USE_SETTLING) ? 1.0 : 0.0;
  const double* y0 = L.y3 + (ni + 1);
  const double* ym = L.y3;
  const double* yp = L.y3 + 2 * (ni + 1);
  for (int i = threadIdx.x; i < ni; i += blockDim.x) {
    double Am, Bm, Cm;
    if (STAGED)
      mol_row_t<double>(row_acc(a, lay, ni, j, i, j - 1, 3), nz, j, i, ysm, ys0, ysp, use_vm, use_set, Am, Bm,
                        Cm);
    else
      mol_row(a, nz, ni, j, i, ysm, ys0, ysp, use_vm, use_set, Am, Bm, Cm);
    double At = eddy[0] + Am;
    double Bt = eddy[1] + Bm;
    double Ct = eddy[2] + Cm;
    L.diff[i] = diffusion_term(a, nz, j, i, flags, At, Bt, Ct, y0[i], ym[i], yp[i]);
    if (want_diag) L.diagd[i] = At;
    if (sup_out && j < nz - 1) sup_out[i] = Bt;
    if (sub_out && j > 0) sub_out[i] = Ct;
  }
}

// Stage-1 assembly: rmod[j] = rhs(y), inv[j] = c0*I - J - diag(diag_d),
// supn[j] = -sup_d, subn[j-1] = -sub_d, with fix_mask (jax_step.py:263-298).
// Latency-bound gathers: four CTAs per SM (the shared-memory limit with the
// drate buffer) beat three without spills (measured on B200, ni=69, nr=1400:
// 4.79 vs 4.89 ms at 296 atmospheres; two per SM: 6.32 ms).
__global__ void __launch_bounds__(LAYER_THREADS, 4)
stage1_kernel(NetDev net, Batch B, const double* __restrict__ y, const double* __restrict__ k,
              const double* __restrict__ dt, const double* __restrict__ atm, int flags,
              const uint8_t* __restrict__ fix_mask, double* __restrict__ ws, const double* __restrict__ adj_v) {
  extern __shared__ double smem[];
  const int b = blockIdx.y, j = blockIdx.x;
  Geo g = geo_of(B, b);
  if (j >= g.nz) return;
  const int ni = B.ni, nz = g.nz;
  LayerSmem L = carve(smem, ni, B.nr, net.T, true);
  AtmRef a = atm_ref(atm + g.atm, nz, ni);
  WsView w = ws_view(ws, g, ni, B.ld);
  const double* yb = y + g.z0 * ni;
  const uint8_t* fm = fix_mask ? fix_mask + g.z0 * ni + (int64_t)j * ni : nullptr;
  const bool adj = adj_v != nullptr;   // J_y blocks of the steady-state adjoint
  const double r = ros2_r();
  const double c0 = adj ? 0.0 : 1.0 / (r * dt[b]);

  __shared__ double coefs[MAX_COEF];
  load_coefs(net, coefs);
  // state row j (the rates; padding slot 1.0) and diag_d of row j, written
  // with the row's diffusion terms by diffusion_rows_kernel ahead of this kernel
  double* yj = L.y3 + (ni + 1);
  for (int t = threadIdx.x; t <= ni; t += blockDim.x) yj[t] = t < ni ? yb[(int64_t)j * ni + t] : 1.0;
  for (int i = threadIdx.x; i < ni; i += blockDim.x) L.diagd[i] = w.aux[(int64_t)j * ni + i];
  __syncthreads();
  layer_rates(net, yj, k + g.z0 * (B.nr + 1) + j, nz, a.M[j], L.rate, L.drate, true);
  __syncthreads();
  // One phase for the species sums and the Jacobian gather: the first 2*ni
  // threads sum a species list, then join the gather on the light end of
  // each rank band. The gather writes each block entry in its final form.
  if (!adj) species_sums(net, coefs, L.rate, L.part);
  double* blk = w.inv + (int64_t)j * ni * B.ld;
  const int ld = B.ld;
  const double bot = (j == 0 && (flags & VB_USE_BOTFLUX)) ? 1.0 : 0.0;
  if (adj) {
    // steady_state_grad.py:153-175: diag = J + diag(A_eddy + A_mol) (+ deposition
    // at the bottom), sup_d = B[:-1], sub_d = C[1:] (no c0, not negated)
    layer_jacobian_each(net, coefs, L.drate, [&](int row, int col, double J) {
      double v = J;
      if (row == col) {
        v = v + L.diagd[row];
        if (j == 0) v = v + (bot != 0.0 ? -a.vdep[row] / a.dzi[0] : 0.0);
      }
      blk[(int64_t)row * ld + col] = v;
    });
    for (int i = threadIdx.x; i < ni; i += blockDim.x)
      w.rmod[(int64_t)j * ni + i] = adj_v[g.z0 * ni + (int64_t)j * ni + i];
    return;
  }
  layer_jacobian_each(net, coefs, L.drate, [&](int row, int col, double J) {
    double v = (row == col ? c0 : 0.0) - J;
    if (row == col) {
      // jax_step.py:283,288: the deposition term joins diag_d before -diag_d is added
      double dd = L.diagd[row];
      if (j == 0) dd = dd + (bot != 0.0 ? -a.vdep[row] / a.dzi[0] : 0.0);
      v = v + (-dd);
    }
    if (fm && fm[row]) v = (row == col) ? c0 : 0.0;
    blk[(int64_t)row * ld + col] = v;
  }, min(2 * ni, (int)blockDim.x));
  __syncthreads();   // the species sums
  for (int i = threadIdx.x; i < ni; i += blockDim.x) {
    // rmod[j] holds the row's diffusion term (diffusion_rows_kernel)
    double v = (L.part[2 * i + 1] - L.part[2 * i]) + w.rmod[(int64_t)j * ni + i];
    if (fm && fm[i]) v = 0.0;
    w.rmod[(int64_t)j * ni + i] = v;
  }
}

// ---------------------------------------------------------------- stage 1, two layers per CTA
// The same assembly as stage1_kernel for layers j0 = 2 blockIdx.x and j0 + 1
// of one atmosphere: every gather word, rate-constant sector and network
// table entry is loaded once for both layers, and each sum runs as two
// independent chains (each in the reference's order, so every value is
// bit-identical to the one-layer kernel's).
constexpr int PAIR_THREADS = 512;

struct PairSmem {
  double* y4;      // [4][ni+1]: layers j0-1 .. j0+2 (padding slot 1.0)
  double* rate;    // [2][nr+1]
  double* drate;   // [2][(nr+1)*T]
  double* diff;    // [2][ni]
  double* diagd;   // [2][ni]
  double* part;    // [2][2*ni]
  double* scal;    // [8]: ysums of the four rows
  double* supb;    // [2][ni]
  double* subb;    // [2][ni]
};

__host__ __device__ inline size_t pair_smem_bytes(int ni, int nr, int T) {
  const size_t d = 4 * (size_t)(ni + 1) + 2 * (size_t)(nr + 1) + 2 * (size_t)(nr + 1) * T + 10 * (size_t)ni + 8 +
                   4 * (size_t)ni;
  return d * sizeof(double);
}

__device__ inline PairSmem carve_pair(double* s, int ni, int nr, int T) {
  PairSmem P;
  P.y4 = s; s += 4 * (ni + 1);
  P.rate = s; s += 2 * (nr + 1);
  P.drate = s; s += 2 * (nr + 1) * T;
  P.diff = s; s += 2 * ni;
  P.diagd = s; s += 2 * ni;
  P.part = s; s += 4 * ni;
  P.scal = s; s += 8;
  P.supb = s; s += 2 * ni;
  P.subb = s;
  return P;
}

// Rates and drates of both layers (rate_slot's expression order per layer).
template <int TT, int RU>
__device__ inline void rates_pair_t(const NetDev& net, const double* y0, const double* y1, const double* kcol,
                                    int64_t kstride, bool two, double M0, double M1, double* rate, double* drate) {
  const int R = net.nr + 1;
  for (int r0 = threadIdx.x; r0 < R; r0 += RU * blockDim.x) {
    double kv[RU][2];
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int r = r0 + u * blockDim.x;
      kv[u][0] = r < R ? __ldcg(kcol + (int64_t)r * kstride) : 0.0;
      kv[u][1] = (two && r < R) ? __ldcg(kcol + (int64_t)r * kstride + 1) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int r = r0 + u * blockDim.x;
      if (r < R) {
        rate_slot<TT>(net, r, y0, kv[u][0], M0, rate, drate, true);
        if (two) rate_slot<TT>(net, r, y1, kv[u][1], M1, rate + R, drate + (int64_t)R * TT, true);
      }
    }
  }
}

__device__ inline void rates_pair(const NetDev& net, const double* y0, const double* y1, const double* kcol,
                                  int64_t kstride, bool two, double M0, double M1, double* rate, double* drate) {
  switch (net.T) {
    case 1: rates_pair_t<1, 3>(net, y0, y1, kcol, kstride, two, M0, M1, rate, drate); return;
    case 2: rates_pair_t<2, 3>(net, y0, y1, kcol, kstride, two, M0, M1, rate, drate); return;
    case 3: rates_pair_t<3, 3>(net, y0, y1, kcol, kstride, two, M0, M1, rate, drate); return;
    case 4: rates_pair_t<4, 3>(net, y0, y1, kcol, kstride, two, M0, M1, rate, drate); return;
    case 5: rates_pair_t<5, 2>(net, y0, y1, kcol, kstride, two, M0, M1, rate, drate); return;
    case 6: rates_pair_t<6, 2>(net, y0, y1, kcol, kstride, two, M0, M1, rate, drate); return;
    case 7: rates_pair_t<7, 2>(net, y0, y1, kcol, kstride, two, M0, M1, rate, drate); return;
    default: rates_pair_t<8, 2>(net, y0, y1, kcol, kstride, two, M0, M1, rate, drate); return;
  }
}

// Loss and production sums of both layers (species_sums' order per layer).
__device__ inline void species_sums_pair(const NetDev& net, const double* coef, const double* rate, double* part) {
  const int R = net.nr + 1;
  for (int t = threadIdx.x; t < 2 * net.ni; t += blockDim.x) {
    const uint2 d = net.sum_desc[t];
    double a0 = 0.0, a1 = 0.0;
    const int e1 = (int)d.x + 32 * (int)d.y;
#pragma unroll 4
    for (int e = (int)d.x; e < e1; e += 32) {
      const uint32_t x = net.sum_w[e];
      const double c = coef[x >> 16];
      const int s = x & 0xffffu;
      a0 = a0 + c * rate[s];
      a1 = a1 + c * rate[R + s];
    }
    part[t] = a0;
    part[2 * net.ni + t] = a1;
  }
}

// Dense Jacobians of both layers (layer_jacobian_each's order and rank bands).
template <typename Store>
__device__ inline void jacobian_pair(const NetDev& net, const double* coef, const double* drate, Store store,
                                     int busy) {
  const int nd = net.ni * net.ni;
  const int64_t D = (int64_t)(net.nr + 1) * net.T;
  const int stride = blockDim.x;
  int q = ((int)threadIdx.x - warp_rotation(busy) % stride + stride) % stride;
  uint2 dn = q < nd ? net.jac_desc[q] : make_uint2(0u, 0u);
  for (; q < nd; q += stride) {
    const uint2 dc = dn;
    if (q + stride < nd) dn = net.jac_desc[q + stride];
    const int e0 = (int)dc.x, e1 = e0 + 32 * (int)(dc.y & 0xffffu);
    double J0 = 0.0, J1 = 0.0;
#pragma unroll 4
    for (int e = e0; e < e1; e += 32) {
      const uint32_t x = net.jac_w[e];
      const double c = coef[x >> 16];
      const int s = x & 0xffffu;
      J0 = J0 + c * drate[s];
      J1 = J1 + c * drate[D + s];
    }
    store((int)((dc.y >> 16) & 0xffu), (int)(dc.y >> 24), J0, J1);
  }
}

// Rates of both layers without drates (the stage-2 right-hand side).
template <int TT>
__device__ inline void rates_pair_rhs_t(const NetDev& net, const double* y0, const double* y1, const double* kcol,
                                        int64_t kstride, bool two, double M0, double M1, double* rate) {
  const int R = net.nr + 1;
  constexpr int RU = 2;
  for (int r0 = threadIdx.x; r0 < R; r0 += RU * blockDim.x) {
    double kv[RU][2];
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int r = r0 + u * blockDim.x;
      kv[u][0] = r < R ? __ldcg(kcol + (int64_t)r * kstride) : 0.0;
      kv[u][1] = (two && r < R) ? __ldcg(kcol + (int64_t)r * kstride + 1) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const int r = r0 + u * blockDim.x;
      if (r < R) {
        rate_slot<TT>(net, r, y0, kv[u][0], M0, rate, nullptr, false);
        if (two) rate_slot<TT>(net, r, y1, kv[u][1], M1, rate + R, nullptr, false);
      }
    }
  }
}

// Stage-2 right-hand side for layers j0 = 2 blockIdx.x and j0 + 1 (the rates
// and species sums of stage2_kernel, gather words shared by the pair; every
// value bit-identical to the one-layer kernel's).
__host__ __device__ inline size_t pair2_smem_bytes(int ni, int nr) {
  return (4 * (size_t)(ni + 1) + 2 * (size_t)(nr + 1) + 8 * (size_t)ni + 8) * sizeof(double);
}

__global__ void __launch_bounds__(PAIR_THREADS, 4)
stage2_pair_kernel(NetDev net, Batch B, const double* __restrict__ y, const double* __restrict__ k,
                   const double* __restrict__ dt, const double* __restrict__ atm, int flags,
                   const uint8_t* __restrict__ fix_mask, double* __restrict__ ws) {
  extern __shared__ double smem[];
  const int b = blockIdx.y, j0 = 2 * blockIdx.x;
  Geo g = geo_of(B, b);
  if (j0 >= g.nz) return;
  const int ni = B.ni, nz = g.nz, R = B.nr + 1;
  const bool two = j0 + 1 < nz;
  double* y4 = smem;
  double* rate = y4 + 4 * (ni + 1);
  double* diff = rate + 2 * R;
  double* part = diff + 2 * ni;
  double* scal = part + 4 * ni;
  AtmRef a = atm_ref(atm + g.atm, nz, ni);
  WsView w = ws_view(ws, g, ni, B.ld);
  const double* yb = y + g.z0 * ni;
  const double r = ros2_r();
  const double dtb = dt[b];
  __shared__ double coefs[MAX_COEF];
  load_coefs(net, coefs);
  // rows j0-1 .. j0+2 of yk2 = y + k1/r (load_rows' expression) and their gas sums
  for (int t = threadIdx.x; t < 4 * (ni + 1); t += blockDim.x) {
    const int wr = t / (ni + 1), i = t % (ni + 1), jj = j0 - 1 + wr;
    double v = 1.0;
    if (i < ni) {
      if (jj >= 0 && jj < nz) {
        v = yb[(int64_t)jj * ni + i];
        v = v + w.k1[(int64_t)jj * ni + i] / r;
      } else {
        v = 0.0;
      }
    }
    y4[t] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int wr = threadIdx.x, jj = j0 - 1 + wr;
    scal[wr] = (jj >= 0 && jj < nz) ? pairwise_sum_masked(y4 + wr * (ni + 1), a.gas, ni) : 0.0;
  }
  __syncthreads();
  for (int l = 0; l < 2; ++l) {
    if (l == 1 && !two) break;
    LayerSmem L;
    L.y3 = y4 + l * (ni + 1);
    L.scal = scal + l;
    L.diff = diff + l * ni;
    L.diagd = nullptr;
    layer_diffusion<2>(a, nz, ni, j0 + l, flags, L, nullptr, nullptr, false, l > 0);
  }
  {
    const double* kcol = k + g.z0 * R + j0;
    const double M0 = a.M[j0], M1 = two ? a.M[j0 + 1] : 0.0;
    switch (net.T) {
      case 1: rates_pair_rhs_t<1>(net, y4 + (ni + 1), y4 + 2 * (ni + 1), kcol, nz, two, M0, M1, rate); break;
      case 2: rates_pair_rhs_t<2>(net, y4 + (ni + 1), y4 + 2 * (ni + 1), kcol, nz, two, M0, M1, rate); break;
      case 3: rates_pair_rhs_t<3>(net, y4 + (ni + 1), y4 + 2 * (ni + 1), kcol, nz, two, M0, M1, rate); break;
      case 4: rates_pair_rhs_t<4>(net, y4 + (ni + 1), y4 + 2 * (ni + 1), kcol, nz, two, M0, M1, rate); break;
      case 5: rates_pair_rhs_t<5>(net, y4 + (ni + 1), y4 + 2 * (ni + 1), kcol, nz, two, M0, M1, rate); break;
      case 6: rates_pair_rhs_t<6>(net, y4 + (ni + 1), y4 + 2 * (ni + 1), kcol, nz, two, M0, M1, rate); break;
      case 7: rates_pair_rhs_t<7>(net, y4 + (ni + 1), y4 + 2 * (ni + 1), kcol, nz, two, M0, M1, rate); break;
      default: rates_pair_rhs_t<8>(net, y4 + (ni + 1), y4 + 2 * (ni + 1), kcol, nz, two, M0, M1, rate); break;
    }
  }
  __syncthreads();
  species_sums_pair(net, coefs, rate, part);
  __syncthreads();
  for (int t = threadIdx.x; t < 2 * ni; t += blockDim.x) {
    const int l = t / ni, i = t - l * ni, j = j0 + l;
    if (l == 1 && !two) break;
    const double* pt = part + l * 2 * ni;
    double v = (pt[2 * i + 1] - pt[2 * i]) + diff[l * ni + i];
    const uint8_t* fm = fix_mask ? fix_mask + g.z0 * ni + (int64_t)j * ni : nullptr;
    if (fm && fm[i]) v = 0.0;
    const double k1v = w.k1[(int64_t)j * ni + i];
    w.rmod[(int64_t)j * ni + i] = v - (2.0 / (r * dtb)) * k1v;
  }
}

__global__ void __launch_bounds__(PAIR_THREADS, 2)
stage1_pair_kernel(NetDev net, Batch B, const double* __restrict__ y, const double* __restrict__ k,
                   const double* __restrict__ dt, const double* __restrict__ atm, int flags,
                   const uint8_t* __restrict__ fix_mask, double* __restrict__ ws) {
  extern __shared__ double smem[];
  const int b = blockIdx.y, j0 = 2 * blockIdx.x;
  Geo g = geo_of(B, b);
  if (j0 >= g.nz) return;
  const int ni = B.ni, nz = g.nz, ld = B.ld;
  const bool two = j0 + 1 < nz;
  PairSmem P = carve_pair(smem, ni, B.nr, net.T);
  AtmRef a = atm_ref(atm + g.atm, nz, ni);
  WsView w = ws_view(ws, g, ni, ld);
  const double* yb = y + g.z0 * ni;
  const double r = ros2_r();
  const double c0 = 1.0 / (r * dt[b]);
  __shared__ double coefs[MAX_COEF];
  load_coefs(net, coefs);
  // rows j0-1 .. j0+2 and their gas sums
  for (int t = threadIdx.x; t < 4 * (ni + 1); t += blockDim.x) {
    const int wr = t / (ni + 1), i = t % (ni + 1), jj = j0 - 1 + wr;
    double v = 1.0;
    if (i < ni) v = (jj >= 0 && jj < nz) ? yb[(int64_t)jj * ni + i] : 0.0;
    P.y4[t] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int wr = threadIdx.x, jj = j0 - 1 + wr;
    P.scal[wr] = (jj >= 0 && jj < nz) ? pairwise_sum_masked(P.y4 + wr * (ni + 1), a.gas, ni) : 0.0;
  }
  __syncthreads();
  // diffusion of each layer (layer_diffusion on a one-layer view of the rows)
  for (int l = 0; l < 2; ++l) {
    if (l == 1 && !two) break;
    LayerSmem L;
    L.y3 = P.y4 + l * (ni + 1);
    L.scal = P.scal + l;
    L.diff = P.diff + l * ni;
    L.diagd = P.diagd + l * ni;
    layer_diffusion(a, nz, ni, j0 + l, flags, L, P.supb + l * ni, P.subb + l * ni, true, l > 0);
  }
  rates_pair(net, P.y4 + (ni + 1), P.y4 + 2 * (ni + 1), k + g.z0 * (B.nr + 1) + j0, nz, two, a.M[j0],
             two ? a.M[j0 + 1] : 0.0, P.rate, P.drate);
  __syncthreads();
  species_sums_pair(net, coefs, P.rate, P.part);
  double* blk0 = w.inv + (int64_t)j0 * ni * ld;
  double* blk1 = blk0 + (int64_t)ni * ld;
  const uint8_t* fm0 = fix_mask ? fix_mask + g.z0 * ni + (int64_t)j0 * ni : nullptr;
  const uint8_t* fm1 = fm0 ? fm0 + ni : nullptr;
  const double bot = (j0 == 0 && (flags & VB_USE_BOTFLUX)) ? 1.0 : 0.0;
  jacobian_pair(net, coefs, P.drate, [&](int row, int col, double J0, double J1) {
    double v = (row == col ? c0 : 0.0) - J0;
    if (row == col) {
      double dd = P.diagd[row];
      if (j0 == 0) dd = dd + (bot != 0.0 ? -a.vdep[row] / a.dzi[0] : 0.0);
      v = v + (-dd);
    }
    if (fm0 && fm0[row]) v = (row == col) ? c0 : 0.0;
    blk0[(int64_t)row * ld + col] = v;
    if (two) {
      double v1 = (row == col ? c0 : 0.0) - J1;
      if (row == col) v1 = v1 + (-P.diagd[ni + row]);
      if (fm1 && fm1[row]) v1 = (row == col) ? c0 : 0.0;
      blk1[(int64_t)row * ld + col] = v1;
    }
  }, min(2 * ni, (int)blockDim.x));
  __syncthreads();   // the species sums
  for (int t = threadIdx.x; t < 2 * ni; t += blockDim.x) {
    const int l = t / ni, i = t - l * ni, j = j0 + l;
    if (l == 1 && !two) break;
    const double* part = P.part + l * 2 * ni;
    const uint8_t* fm = l ? fm1 : fm0;
    double v = (part[2 * i + 1] - part[2 * i]) + P.diff[l * ni + i];
    const bool fixed = fm && fm[i];
    if (fixed) v = 0.0;
    w.rmod[(int64_t)j * ni + i] = v;
    if (j < nz - 1) {
      double s2 = -P.supb[l * ni + i];
      if (fixed) s2 = 0.0;
      w.supn[(int64_t)j * ni + i] = s2;
    }
    if (j > 0) {
      double s2 = -P.subb[l * ni + i];
      if (fixed) s2 = 0.0;
      w.subn[(int64_t)(j - 1) * ni + i] = s2;
    }
  }
}

// Stage-2 right-hand side: rmod[j] = rhs(yk2) - 2/(r dt) k1[j] with
// yk2 = y + k1/r (jax_step.py:303-310). No drate buffer, so eight CTAs fit an
// SM; occupancy, not per-thread ILP, hides the gathers' latency (measured on
// B200, ni=69, nr=1400, 296 atmospheres: 3 / 4 / 5 / 6 CTAs per SM 2.22 /
// 1.87 / 1.70 / 1.57 ms; 8 with rate constants loaded 2 deep instead of 6:
// 1.53 ms, despite the spills at 32 registers).
__global__ void __launch_bounds__(LAYER_THREADS, 8)
stage2_kernel(NetDev net, Batch B, const double* __restrict__ y, const double* __restrict__ k,
              const double* __restrict__ dt, const double* __restrict__ atm, int flags,
              const uint8_t* __restrict__ fix_mask, double* __restrict__ ws, double* __restrict__ resid) {
  extern __shared__ double smem[];
  const int b = blockIdx.y, j = blockIdx.x;
  Geo g = geo_of(B, b);
  if (j >= g.nz) return;
  const int ni = B.ni, nz = g.nz;
  LayerSmem L = carve(smem, ni, B.nr, net.T, false);
  AtmRef a = atm_ref(atm + g.atm, nz, ni);
  WsView w = ws_view(ws, g, ni, B.ld);
  const double* yb = y + g.z0 * ni;
  const uint8_t* fm = fix_mask ? fix_mask + g.z0 * ni + (int64_t)j * ni : nullptr;
  const double r = ros2_r();
  const bool res = resid != nullptr;   // steady-state residual f(y) (steady_state_grad.py:116-130)
  const double dtb = res ? 1.0 : dt[b];

  __shared__ double coefs[MAX_COEF];
  load_coefs(net, coefs);
  // state row j (yk2 = y + k1/r, load_rows' expression; padding slot 1.0)
  double* yj = L.y3 + (ni + 1);
  for (int t = threadIdx.x; t <= ni; t += blockDim.x) {
    double v = 1.0;
    if (t < ni) {
      v = yb[(int64_t)j * ni + t];
      if (!res) v = v + w.k1[(int64_t)j * ni + t] / r;
    }
    yj[t] = v;
  }
  __syncthreads();
  layer_rates(net, yj, k + g.z0 * (B.nr + 1) + j, nz, a.M[j], L.rate, nullptr, false);
  __syncthreads();
  species_sums(net, coefs, L.rate, L.part);
  __syncthreads();
  // rmod[j] (resid[j]) holds the row's diffusion term (diffusion_rows_kernel)
  const double* dif = res ? resid + g.z0 * ni : w.rmod;
  for (int i = threadIdx.x; i < ni; i += blockDim.x) {
    double v = (L.part[2 * i + 1] - L.part[2 * i]) + dif[(int64_t)j * ni + i];
    if (res) {
      resid[g.z0 * ni + (int64_t)j * ni + i] = v;
      continue;
    }
    if (fm && fm[i]) v = 0.0;
    double k1v = w.k1[(int64_t)j * ni + i];
    w.rmod[(int64_t)j * ni + i] = v - (2.0 / (r * dtb)) * k1v;
  }
}

// Standalone chemistry: dydt (and optionally the Jacobian) of a uniform batch.
__global__ void __launch_bounds__(LAYER_THREADS)
chem_kernel(NetDev net, int nz, const double* __restrict__ y, const double* __restrict__ M,
            const double* __restrict__ k, double* __restrict__ dydt, double* __restrict__ jac) {
  extern __shared__ double smem[];
  const int b = blockIdx.y, j = blockIdx.x;
  const int ni = net.ni;
  bool want_jac = jac != nullptr;
  LayerSmem L = carve(smem, ni, net.nr, net.T, want_jac, want_jac);
  const double* yrow = y + ((int64_t)b * nz + j) * ni;
  __shared__ double coefs[MAX_COEF];
  load_coefs(net, coefs);
  for (int i = threadIdx.x; i <= ni; i += blockDim.x) L.y3[i] = i < ni ? yrow[i] : 1.0;
  __syncthreads();
  layer_rates(net, L.y3, k + (int64_t)b * (net.nr + 1) * nz + j, nz, M[(int64_t)b * nz + j], L.rate,
              L.drate, want_jac);
  __syncthreads();
  species_sums(net, coefs, L.rate, L.part);
  if (want_jac) layer_jacobian(net, coefs, L.drate, L.jac);
  __syncthreads();
  if (dydt)
    for (int i = threadIdx.x; i < ni; i += blockDim.x)
      dydt[((int64_t)b * nz + j) * ni + i] = L.part[2 * i + 1] - L.part[2 * i];
  if (want_jac) {
    double* out = jac + ((int64_t)b * nz + j) * ni * ni;
    for (int d = threadIdx.x; d < ni * ni; d += blockDim.x) out[d] = L.jac[d];
  }
}

// Standalone diffusion of a uniform batch (jax_step.py:67-246).
__global__ void __launch_bounds__(LAYER_THREADS)
diffusion_kernel(int nz, int ni, const double* __restrict__ y, const double* __restrict__ atm,
                 int flags, double* __restrict__ diff, double* __restrict__ diag_d,
                 double* __restrict__ sup_d, double* __restrict__ sub_d) {
  extern __shared__ double smem[];
  const int b = blockIdx.y, j = blockIdx.x;
  LayerSmem L = carve(smem, ni, 0, 1, false);
  AtmRef a = atm_ref(atm + (int64_t)b * VB_ATM_DOUBLES(nz, ni), nz, ni);
  const double* yb = y + (int64_t)b * nz * ni;
  load_rows<true>(yb, nullptr, a.gas, nz, ni, j, 1.0, false, L);
  __syncthreads();
  double* supo = sup_d ? sup_d + ((int64_t)b * (nz - 1) + j) * ni : nullptr;
  double* subo = sub_d ? sub_d + ((int64_t)b * (nz - 1) + (j - 1)) * ni : nullptr;
  layer_diffusion(a, nz, ni, j, flags, L, supo, subo, true);
  __syncthreads();
  for (int i = threadIdx.x; i < ni; i += blockDim.x) {
    if (diff) diff[((int64_t)b * nz + j) * ni + i] = L.diff[i];
    if (diag_d) {
      double dd = L.diagd[i];
      if (j == 0) dd = dd + ((flags & VB_USE_BOTFLUX) ? -a.vdep[i] / a.dzi[0] : 0.0);
      diag_d[((int64_t)b * nz + j) * ni + i] = dd;
    }
  }
}

// ---------------------------------------------------------------- diffusion rows ahead of the stages
// The eddy + molecular diffusion of every layer (the same functions on the
// same inputs as layer_diffusion, so the same bits), computed ahead of the
// stage kernels, whose heavy per-layer CTAs then load one state row and no
// atmosphere fields. One CTA per block of DIFF_LAYERS consecutive layers of
// one atmosphere: the block's state rows, their gas sums, per-layer fields
// and eddy coefficients are formed once, then every (layer, species) item of
// the block runs in parallel.
//   mode 0 (stage 1):  rmod[j] = diff, aux[j] = diag_d, supn[j] = -sup_d,
//                      subn[j-1] = -sub_d (0 on fixed species);
//   mode 1 (stage 1 of the adjoint): aux[j] = diag_d, supn[j] = sup_d,
//                      subn[j-1] = sub_d (steady_state_grad.py:153-175);
//   mode 2 (stage 2):  rmod[j] = diff at yk2 = y + k1/r (with resid: resid[j]
//                      = diff at y, the residual; ws unused).
// Four CTAs per SM (64 registers, 32 bytes spilled): 0.239 ms per launch at
// 296 config-0 atmospheres on B200 against 0.261 with three (74 registers);
// the items are chains of FP64 divisions, hidden by resident warps.
constexpr int DIFF_THREADS = 256;
constexpr int DIFF_LAYERS = 8;
__host__ __device__ inline size_t diff_block_smem_bytes(int ni) {
  constexpr int NR = DIFF_LAYERS + 2;
  return ((size_t)NR * (ni + 1) + ni + NR + 7 * NR + 3 * DIFF_LAYERS) * sizeof(double);
}

__global__ void __launch_bounds__(DIFF_THREADS, 4)
diffusion_rows_kernel(Batch B, const double* __restrict__ y, const double* __restrict__ atm, int flags,
                      const uint8_t* __restrict__ fix_mask, double* __restrict__ ws, double* __restrict__ resid,
                      int mode) {
  extern __shared__ double smem[];
  constexpr int LB = DIFF_LAYERS, NR = LB + 2;
  const int b = blockIdx.y, jb = blockIdx.x * LB;
  Geo g = geo_of(B, b);
  if (jb >= g.nz) return;
  const int ni = B.ni, nz = g.nz, rs = ni + 1;
  double* ys = smem;               // [NR][ni+1]: rows jb-1 .. jb+LB (0 outside [0, nz); padding 1.0)
  double* gas = ys + NR * rs;      // [ni]
  double* scal = gas + ni;         // [NR]: gas sums of those rows
  double* lay = scal + NR;         // [7][NR]: Kzz dzi vz Hpi Ti Tco g of those layers
  double* edd = lay + 7 * NR;      // [LB][3]: eddy A, B, C of the block's layers
  const AtmRef a = atm_ref(atm + g.atm, nz, ni);
  const WsView w = ws_view(ws, g, ni, B.ld);
  const double* yb = y + g.z0 * ni;
  const bool yk2 = mode == 2 && !resid;   // stage 2: rows of yk2 = y + k1/r (load_rows' expression)
  const double r = ros2_r();
  for (int t = threadIdx.x; t < NR * rs; t += blockDim.x) {
    const int rr = t / rs, i = t % rs, jj = jb - 1 + rr;
    double v = 1.0;
    if (i < ni) {
      if (jj >= 0 && jj < nz) {
        v = yb[(int64_t)jj * ni + i];
        if (yk2) v = v + w.k1[(int64_t)jj * ni + i] / r;
      } else {
        v = 0.0;
      }
    }
    ys[t] = v;
  }
  for (int i = threadIdx.x; i < ni; i += blockDim.x) gas[i] = a.gas[i];
  for (int t = threadIdx.x; t < 7 * NR; t += blockDim.x) {
    const int f = t / NR, m = jb - 1 + t % NR;
    const double* src = f == 0 ? a.Kzz : f == 1 ? a.dzi : f == 2 ? a.vz : f == 3 ? a.Hpi : f == 4 ? a.Ti
                      : f == 5 ? a.Tco : a.g;
    lay[t] = (m >= 0 && m < nz) ? src[m] : 0.0;
  }
  __syncthreads();
  if (threadIdx.x < NR) {
    const int jj = jb - 1 + (int)threadIdx.x;
    scal[threadIdx.x] = (jj >= 0 && jj < nz) ? pairwise_sum_masked(ys + threadIdx.x * rs, gas, ni) : 0.0;
  }
  __syncthreads();
  if (threadIdx.x < LB) {
    const int l = threadIdx.x, j = jb + l;
    if (j < nz) {
      RowAcc E{};
      E.lay = lay;
      E.j0 = j - 1;
      E.base = jb - 1;
      E.S = NR;
      double A, Bc, C;
      eddy_row_t<double>(E, nz, j, scal[l], scal[l + 1], scal[l + 2], A, Bc, C);
      edd[3 * l] = A;
      edd[3 * l + 1] = Bc;
      edd[3 * l + 2] = C;
    }
  }
  __syncthreads();
  const double use_vm = (flags & VB_USE_VM_MOL) ? 1.0 : 0.0;
  const double use_set = (flags & VB_USE_SETTLING) ? 1.0 : 0.0;
  for (int q = threadIdx.x; q < LB * ni; q += blockDim.x) {
    const int l = q / ni, i = q % ni, j = jb + l;
    if (j >= nz) continue;
    double Am, Bm, Cm;
    mol_row_t<double>(row_acc(a, lay, ni, j, i, jb - 1, NR), nz, j, i, scal[l], scal[l + 1], scal[l + 2], use_vm,
                      use_set, Am, Bm, Cm);
    const double At = edd[3 * l] + Am;
    const double Bt = edd[3 * l + 1] + Bm;
    const double Ct = edd[3 * l + 2] + Cm;
    const double d = diffusion_term(a, nz, j, i, flags, At, Bt, Ct, ys[(l + 1) * rs + i], ys[l * rs + i],
                                    ys[(l + 2) * rs + i]);
    if (mode == 2) {
      (resid ? resid + g.z0 * ni : w.rmod)[(int64_t)j * ni + i] = d;
      continue;
    }
    if (mode == 0) w.rmod[(int64_t)j * ni + i] = d;
    w.aux[(int64_t)j * ni + i] = At;
    const bool fixed = mode == 0 && fix_mask && fix_mask[g.z0 * ni + (int64_t)j * ni + i];
    if (j < nz - 1) w.supn[(int64_t)j * ni + i] = mode == 1 ? Bt : (fixed ? 0.0 : -Bt);
    if (j > 0) w.subn[(int64_t)(j - 1) * ni + i] = mode == 1 ? Ct : (fixed ? 0.0 : -Ct);
  }
}

static cudaError_t launch_diffusion_rows(const Batch& B, const double* y, const double* atm, int flags,
                                         const uint8_t* fm, double* ws, double* resid, int mode, cudaStream_t st) {
  dim3 grid((B.nz + DIFF_LAYERS - 1) / DIFF_LAYERS, B.count);
  diffusion_rows_kernel<<<grid, DIFF_THREADS, diff_block_smem_bytes(B.ni), st>>>(B, y, atm, flags, fm, ws, resid,
                                                                                 mode);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- layer-vectorized stage 2
// The stage-2 right-hand side with one thread per layer instead of one CTA per
// layer: every term of a species list is then one coalesced load of a row of
// layers that the whole warp shares, in place of a dependent chain of table,
// shared-memory and L2 loads per lane. Two passes:
//  * lv_rates_kernel: the rate of every reaction slot at every layer of an
//    atmosphere at yk2 = y + k1/r (the state rows staged transposed in shared
//    memory; the rate constants k[r][z] read with the layers contiguous, the
//    reference's layout), into the rate region (rows [nr+1][nz_b]);
//  * lv_sums_kernel (a CTA per species and atmosphere, a thread per layer):
//    the species' loss and production sums, rmod = rhs(yk2) - 2/(r dt) k1.
// Each sum runs over the same terms, in the same order, with the same
// operations as in stage2_kernel, so the results are identical. (The same
// scheme for stage 1, with the rate derivatives staged too and the Jacobian
// rows summed per layer, measured slower than stage1_kernel on B200: 3.0 ms
// against 2.5 at 296 config-0 atmospheres; its scattered block-row stores
// and staging buffers cost more than the per-layer gathers.)
constexpr int LV_LAYERS = 128;         // layers of one thread group (a z-tile)
constexpr int LV_RATE_THREADS = 512;   // four groups; reactions dealt round the groups

__host__ __device__ inline size_t lv_rates_smem_bytes(int ni) {
  return (size_t)(ni + 1) * (LV_LAYERS + 1) * sizeof(double);
}

template <int TT>
__global__ void __launch_bounds__(LV_RATE_THREADS)
lv_rates_kernel(NetDev net, Batch B, const double* __restrict__ y, const double* __restrict__ k,
                const double* __restrict__ atm, double* __restrict__ ws) {
  extern __shared__ double smem[];
  constexpr int RU = 4;   // rate constants loaded ahead
  const int b = blockIdx.y;
  const Geo g = geo_of(B, b);
  const int ni = B.ni, nzb = g.nz, R = B.nr + 1, S = LV_LAYERS + 1;
  const int r_lo = (int)((int64_t)R * blockIdx.x / gridDim.x);
  const int r_hi = (int)((int64_t)R * (blockIdx.x + 1) / gridDim.x);
  const double* yb = y + g.z0 * ni;
  const WsView w = ws_view(ws, g, ni, B.ld);
  const AtmRef a = atm_ref(atm + g.atm, nzb, ni);
  const double* kb = k + g.z0 * R;
  double* rate = B.rates + g.z0 * rates_region_doubles(B.nr);
  const double r = ros2_r();
  const int grp = threadIdx.x / LV_LAYERS, zl = threadIdx.x % LV_LAYERS, ngrp = blockDim.x / LV_LAYERS;
  double* yT = smem;   // [ni+1][S]: yk2 of species i at layer zl (row ni: the padding slot, 1.0)
  for (int zt = 0; zt < nzb; zt += LV_LAYERS) {
    const int nzt = min(LV_LAYERS, nzb - zt);
    __syncthreads();   // the previous tile's reads
    for (int e = threadIdx.x; e < nzt * ni; e += blockDim.x) {
      const int zz = e / ni, i = e - zz * ni;
      const int64_t q = (int64_t)(zt + zz) * ni + i;
      yT[i * S + zz] = yb[q] + w.k1[q] / r;   // stage2_kernel's expression
    }
    for (int zz = threadIdx.x; zz < LV_LAYERS; zz += blockDim.x) yT[ni * S + zz] = 1.0;
    __syncthreads();
    const int z = zt + zl;
    const bool on = zl < nzt;
    const double M = on ? a.M[z] : 0.0;
    for (int r0 = r_lo + grp; r0 < r_hi; r0 += RU * ngrp) {
      double kv[RU];
#pragma unroll
      for (int u = 0; u < RU; ++u) {
        const int rr = r0 + u * ngrp;
        kv[u] = (on && rr < r_hi) ? __ldcg(kb + (int64_t)rr * nzb + z) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < RU; ++u) {
        const int rr = r0 + u * ngrp;
        if (rr < r_hi) {
          double yr[TT], st[TT], d[TT];
#pragma unroll
          for (int s = 0; s < TT; ++s) {
            st[s] = net.r_st[rr * TT + s];
            yr[s] = yT[net.r_idx[rr * TT + s] * S + zl];
          }
          const double rt = rate_terms<TT>(yr, st, kv[u], M, net.three[rr] != 0, false, d);
          if (on) rate[(int64_t)rr * nzb + z] = rt;
        }
      }
    }
  }
}

__global__ void __launch_bounds__(LV_LAYERS)
lv_sums_kernel(NetDev net, Batch B, const double* __restrict__ dt, const uint8_t* __restrict__ fix_mask,
               double* __restrict__ ws) {
  __shared__ double coefs[MAX_COEF];
  load_coefs(net, coefs);
  __syncthreads();
  const int i = blockIdx.x, b = blockIdx.y;
  const Geo g = geo_of(B, b);
  const int ni = B.ni, nzb = g.nz;
  const WsView w = ws_view(ws, g, ni, B.ld);
  const double* rate = B.rates + g.z0 * rates_region_doubles(B.nr);
  const double r = ros2_r();
  for (int zt = 0; zt < nzb; zt += LV_LAYERS) {
    const int z = zt + (int)threadIdx.x;
    if (z >= nzb) break;
    double part[2];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int e0 = net.sum_nptr[2 * i + t], e1 = net.sum_nptr[2 * i + t + 1];
      double acc = 0.0;
#pragma unroll 8
      for (int e = e0; e < e1; ++e) {
        const uint32_t x = net.sum_nw[e];
        acc = acc + coefs[x >> 16] * rate[(int64_t)(x & 0xffffu) * nzb + z];
      }
      part[t] = acc;
    }
    // rmod holds the row's diffusion term (diffusion_rows_kernel)
    const int64_t q = (int64_t)z * ni + i;
    double v = (part[1] - part[0]) + w.rmod[q];
    if (fix_mask && fix_mask[g.z0 * ni + q]) v = 0.0;
    w.rmod[q] = v - (2.0 / (r * dt[b])) * w.k1[q];
  }
}

// Reaction chunks per atmosphere of lv_rates_kernel: about two waves of
// three 512-thread CTAs per SM, at least 8 reaction slots per chunk.
static int lv_rate_chunks(const Batch& B) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
    sms = 148;
  const int want = (6 * sms + B.count - 1) / B.count;
  return std::max(1, std::min(want, (B.nr + 1) / 8));
}

static cudaError_t launch_lv_stage2(const NetDev& net, const Batch& B, const double* y, const double* k,
                                    const double* dt, const double* atm, const uint8_t* fm, double* ws,
                                    cudaStream_t st) {
  const size_t sm = lv_rates_smem_bytes(B.ni);
  dim3 grid(lv_rate_chunks(B), B.count);
  cudaError_t e = cudaSuccess;
  auto go = [&](auto kern) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) kern<<<grid, LV_RATE_THREADS, sm, st>>>(net, B, y, k, atm, ws);
  };
  switch (net.T) {
    case 1: go(lv_rates_kernel<1>); break;
    case 2: go(lv_rates_kernel<2>); break;
    case 3: go(lv_rates_kernel<3>); break;
    case 4: go(lv_rates_kernel<4>); break;
    case 5: go(lv_rates_kernel<5>); break;
    case 6: go(lv_rates_kernel<6>); break;
    case 7: go(lv_rates_kernel<7>); break;
    default: go(lv_rates_kernel<8>); break;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  lv_sums_kernel<<<dim3(B.ni, B.count), LV_LAYERS, 0, st>>>(net, B, dt, fm, ws);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- launchers
// Stage-1 / stage-2 kernels of the Ros2 step (VbTuning.stage1_layers): one
// layer per CTA by default (measured on B200 at 296 config-0 atmospheres, the
// two-layer kernels make the step 13.08 ms against 12.81: the gather latency
// is hidden better by more resident CTAs than by two chains per thread).
static constexpr int kStage1DefaultLayers = 1;

cudaError_t launch_stage1(const NetDev& net, const Batch& B, const double* y, const double* k,
                          const double* dt, const double* atm, int flags, const uint8_t* fm, double* ws,
                          cudaStream_t st, const double* adj_v) {
  const int layers = B.stage1_layers ? B.stage1_layers : kStage1DefaultLayers;
  if (!adj_v && layers == 2) {
    size_t sm = pair_smem_bytes(B.ni, B.nr, net.T);
    cudaError_t e = cudaFuncSetAttribute(stage1_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((B.nz + 1) / 2, B.count);
    stage1_pair_kernel<<<grid, PAIR_THREADS, sm, st>>>(net, B, y, k, dt, atm, flags, fm, ws);
    return cudaGetLastError();
  }
  cudaError_t e = launch_diffusion_rows(B, y, atm, flags, fm, ws, nullptr, adj_v ? 1 : 0, st);
  if (e != cudaSuccess) return e;
  size_t sm = layer_smem_bytes(B.ni, B.nr, net.T, true);
  cudaFuncSetAttribute(stage1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 grid(B.nz, B.count);
  stage1_kernel<<<grid, LAYER_THREADS, sm, st>>>(net, B, y, k, dt, atm, flags, fm, ws, adj_v);
  return cudaGetLastError();
}

cudaError_t launch_stage2(const NetDev& net, const Batch& B, const double* y, const double* k,
                          const double* dt, const double* atm, int flags, const uint8_t* fm, double* ws,
                          cudaStream_t st, double* resid) {
  const int layers = B.stage1_layers ? B.stage1_layers : kStage1DefaultLayers;
  if (B.rates && !resid && layers != 2) {
    cudaError_t e = launch_diffusion_rows(B, y, atm, flags, fm, ws, nullptr, 2, st);
    if (e == cudaSuccess) e = launch_lv_stage2(net, B, y, k, dt, atm, fm, ws, st);
    return e;
  }
  if (!resid && layers == 2) {
    size_t sm = pair2_smem_bytes(B.ni, B.nr);
    cudaError_t e = cudaFuncSetAttribute(stage2_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((B.nz + 1) / 2, B.count);
    stage2_pair_kernel<<<grid, PAIR_THREADS, sm, st>>>(net, B, y, k, dt, atm, flags, fm, ws);
    return cudaGetLastError();
  }
  cudaError_t e = launch_diffusion_rows(B, y, atm, flags, fm, ws, resid, 2, st);
  if (e != cudaSuccess) return e;
  size_t sm = layer_smem_bytes(B.ni, B.nr, net.T, false);
  cudaFuncSetAttribute(stage2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 grid(B.nz, B.count);
  stage2_kernel<<<grid, LAYER_THREADS, sm, st>>>(net, B, y, k, dt, atm, flags, fm, ws, resid);
  return cudaGetLastError();
}

cudaError_t launch_chem(const NetDev& net, int batch, int nz, const double* y, const double* M,
                        const double* k, double* dydt, double* jac, cudaStream_t st) {
  size_t sm = layer_smem_bytes(net.ni, net.nr, net.T, jac != nullptr, jac != nullptr);
  cudaFuncSetAttribute(chem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 grid(nz, batch);
  chem_kernel<<<grid, LAYER_THREADS, sm, st>>>(net, nz, y, M, k, dydt, jac);
  return cudaGetLastError();
}

cudaError_t launch_diffusion(int batch, int nz, int ni, const double* y, const double* atm, int flags,
                             double* diff, double* diag_d, double* sup_d, double* sub_d,
                             cudaStream_t st) {
  size_t sm = layer_smem_bytes(ni, 0, 1, false);
  dim3 grid(nz, batch);
  diffusion_kernel<<<grid, LAYER_THREADS, sm, st>>>(nz, ni, y, atm, flags, diff, diag_d, sup_d, sub_d);
  return cudaGetLastError();
}

}  // namespace vb
