// Shared device-side definitions of the B200 Ros2 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vulcan_b200.h"

namespace vb {

// Device-resident network tables (reference chem.py:28-80 plus gather tables).
struct NetDev {
  int ni, nr, T;                 // species, reaction slots (rows nr+1), max_terms
  const int32_t* r_idx;          // [nr+1][T]
  const int32_t* p_idx;          // [nr+1][T]
  const double* r_st;            // [nr+1][T]
  const double* p_st;            // [nr+1][T]
  const uint8_t* three;          // [nr+1]
  // Gather tables, one 32-bit word per term: the low 16 bits index a rate
  // (loss / prod: reaction r) or a drate slot (Jacobian: r*T+s), the high 16
  // bits a coefficient in coef_tab (the distinct stoichiometries, <= 256).
  // RHS: list t = 2 i (loss) or 2 i + 1 (production) of species i, the
  // (r*T+s) slots whose reactant (loss) or product index is i, in increasing
  // flat order (segment_sum order); the coefficient is r_st[r*T+s] or
  // p_st[r*T+s]. The words of each group of 32 consecutive lists are
  // interleaved (term k of list t at its first word + 32 k), so the lanes of
  // a warp summing lists t = 32 g .. 32 g + 31 load one line per term.
  const uint2* sum_desc;         // [2 ni]: {first word in sum_w, term count}
  const uint32_t* sum_w;
  // Jacobian: for destination d = row*ni+col, the contributions (r, o, s) in
  // increasing flat order (r*2T + o)*T + s (chem.py:193-207 scatter order);
  // the coefficient is -r_st[r][o] (o < T) or p_st[r][o-T]. jac_ptr is the
  // CSR of that order; jac_w holds the words interleaved by groups of 32
  // consecutive ranks of jac_desc (term i of a rank at its first word + 32 i).
  const int32_t* jac_ptr;        // [ni*ni+1]
  const uint32_t* jac_w;
  const double* coef_tab;        // [n_coef]
  int n_coef;
  // Destinations in decreasing term count: {first term in jac_w,
  // count | row << 16 | col << 24}.
  const uint2* jac_desc;         // [ni*ni]
  // The species lists in natural order, for the layer-vectorized stage 2
  // (one thread per layer, every term of a list read by the whole warp):
  // list t (2 i loss, 2 i + 1 production) at sum_nw[sum_nptr[t] .. sum_nptr[t+1]).
  const int32_t* sum_nptr;       // [2 ni + 1]
  const uint32_t* sum_nw;
};

constexpr int LAYER_THREADS = 256;
constexpr int MAX_COEF = 256;   // distinct stoichiometric coefficients of a network

// Term word of a gather table: index (low 16 bits) and coefficient id.
__host__ __device__ __forceinline__ uint32_t term_word(int idx, int cid) {
  return (uint32_t)idx | ((uint32_t)cid << 16);
}

// Offsets (in doubles) of the fields of one atmosphere in the atm blob.
struct AtmOff {
  int64_t Kzz, dzi, vz, Hpi, Ti, Tco, g, M, Dzz, vm, vs, ms, alpha, top, bot, vdep, gas;
};

__host__ __device__ inline AtmOff atm_offsets(int nz, int ni) {
  AtmOff o;
  int64_t NZ = nz, NI = ni;
  o.Kzz = 0; o.dzi = NZ; o.vz = 2 * NZ; o.Hpi = 3 * NZ; o.Ti = 4 * NZ; o.Tco = 5 * NZ;
  o.g = 6 * NZ; o.M = 7 * NZ;
  o.Dzz = 8 * NZ; o.vm = o.Dzz + NZ * NI; o.vs = o.vm + NZ * NI;
  o.ms = o.vs + NZ * NI; o.alpha = o.ms + NI; o.top = o.alpha + NI; o.bot = o.top + NI;
  o.vdep = o.bot + NI; o.gas = o.vdep + NI;
  return o;
}

// Per-atmosphere geometry of a (possibly ragged) batch.
struct Batch {
  int count;          // atmospheres
  int nz;             // layers (uniform) or maximum layers (ragged)
  int ni;
  int nr;             // reaction slots (k has nr+1 rows)
  int ld;             // row stride of stored inverse blocks (ni rounded up to even)
  const int64_t* zoff;  // [count+1] prefix sums of layers, or nullptr (uniform)
  // launch shapes chosen by the network's tuning (VbTuning; 0 = automatic)
  int factor_kernel = 0;   // 1 blocked tensor-core, 2 scalar Gauss-Jordan, 3 pipelined
  int factor_ctas = 0;     // CTAs per SM of the factor (1 or 2, where both fit)
  int sweep_stages = 0;    // bulk-copy ring depth of the sweeps (1..3)
  int stage1_layers = 0;   // layers per stage-1 CTA (1 or 2)
  // rate region of the layer-vectorized stage 2 (rates_region_doubles per
  // layer), or nullptr: the per-layer stage-2 kernel
  double* rates = nullptr;
};

// Doubles per layer of the rate region: the rate of every reaction slot, rows
// [nr+1][nz_b] per atmosphere (layers contiguous).
__host__ __device__ inline int64_t rates_region_doubles(int nr) { return (int64_t)nr + 1; }

struct Geo {
  int nz;
  int64_t z0;        // first layer of this atmosphere in the packed layer axis
  int64_t atm;       // blob offset (doubles)
  int64_t ws;        // workspace offset (doubles)
};

// Workspace doubles per layer: inverse block + rmod + k1 + sup_neg + sub_neg +
// spare, rounded up to 16 doubles so every atmosphere's blocks start on a
// 128-byte boundary (bulk copies need 16-byte aligned addresses and sizes).
__host__ __device__ inline int64_t ws_per_layer(int ni, int ld) {
  return (((int64_t)ni * ld + 5 * (int64_t)ni) + 15) & ~(int64_t)15;
}

__device__ __forceinline__ Geo geo_of(const Batch& B, int b) {
  Geo g;
  if (B.zoff) {
    g.z0 = B.zoff[b];
    g.nz = (int)(B.zoff[b + 1] - g.z0);
  } else {
    g.z0 = (int64_t)b * B.nz;
    g.nz = B.nz;
  }
  g.atm = g.z0 * (8 + 3 * (int64_t)B.ni) + (int64_t)b * 6 * B.ni;
  g.ws = g.z0 * ws_per_layer(B.ni, B.ld);
  return g;
}

// Workspace sub-arrays of one atmosphere (all doubles).
struct WsView {
  double* inv;   // [nz][ni][ld]
  double* rmod;  // [nz][ni]  forward-eliminated right-hand side
  double* k1;    // [nz][ni]
  double* supn;  // [nz][ni]  (first nz-1 rows used): negated super-diagonal (solver's sup_d)
  double* subn;  // [nz][ni]  negated sub-diagonal (solver's sub_d)
  double* aux;   // [nz][ni]
};

__device__ __forceinline__ WsView ws_view(double* ws, const Geo& g, int ni, int ld) {
  WsView v;
  v.inv = ws + g.ws;
  int64_t blk = (int64_t)g.nz * ni * ld;
  int64_t vec = (int64_t)g.nz * ni;
  v.rmod = v.inv + blk;
  v.k1 = v.rmod + vec;
  v.supn = v.k1 + vec;
  v.subn = v.supn + vec;
  v.aux = v.subn + vec;
  return v;
}

__host__ __device__ inline int round_even(int n) { return (n + 1) & ~1; }

// ---- mixed-precision region of the Ros2 step (after the FP64 workspace):
// per atmosphere, [nz][ni][ldf] FP32 inverses of the row-equilibrated
// eliminated blocks (ldf = ni rounded up to 4, so each block is a multiple of
// 16 bytes), then [nz][ni] row scales r (A'^{-1} = X diag(r)), then [nz][ni]
// scratch (the forward-eliminated residual of a refinement pass).
__host__ __device__ inline int round4(int n) { return (n + 3) & ~3; }
__host__ __device__ inline int64_t mx_bytes_per_layer(int ni) {
  return (int64_t)ni * round4(ni) * 4 + 16 * (int64_t)ni;
}
struct MxView {
  float* X;      // [nz][ni][ldf]
  double* rs;    // [nz][ni]
  double* tmp;   // [nz][ni]
};
__host__ __device__ inline MxView mx_view(void* mx, int64_t z0, int nz, int ni) {
  char* base = static_cast<char*>(mx) + z0 * mx_bytes_per_layer(ni);
  MxView v;
  v.X = reinterpret_cast<float*>(base);
  v.rs = reinterpret_cast<double*>(base + (int64_t)nz * ni * round4(ni) * 4);
  v.tmp = v.rs + (int64_t)nz * ni;
  return v;
}

// ---------------------------------------------------------------- bulk copies
// Global -> shared bulk copies (cp.async.bulk, no multicast) completed on an
// mbarrier. Every wait is bounded: a wait that gives up reports false and the
// caller sets VB_STATUS_WATCHDOG.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
  for (long long it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
constexpr long long WAIT_LIMIT = 1ll << 22;

// mbarriers as intra-CTA producer/consumer signals (no async copies): an
// arrival (release) per producing thread, a bounded wait (acquire) that also
// gives up as soon as another warp has raised *abort.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t parity, long long limit,
                                                   const volatile int* abort) {
  for (long long it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (*abort) return false;
  }
  return false;
}

// Ros2 constants (reference jax_step.py:257-258).
__device__ __forceinline__ double ros2_r() { return 1.0 + 1.0 / sqrt(2.0); }

}  // namespace vb
