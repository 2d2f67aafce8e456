// Block-tridiagonal Thomas for dense diagonal blocks and diagonal off-diagonal
// blocks (reference solver.py:33-126), one persistent CTA per atmosphere.
//
// factor: for each layer j (serial in z)
//     A'_j  = D_j - (sub_d[j-1] sup_d[j-1]^T) o A'_{j-1}^{-1}     (solver.py:47)
//     Inv_j = A'_j^{-1}                                            (solver.py:46,48)
// Each A'_j is inverted in place by Gauss-Jordan elimination with threshold
// partial pivoting (pivot_key32) on a register-resident tile (implicit
// pivoting: no row exchanges),
// one serial chain of ni pivot steps per layer with one block barrier each.
// The forward sweep of the first right-hand side rides along
// (solver.py:73-88). The stored inverses turn every later solve into
// matrix-vector products (solver.py:91-111).
#include <cuda_runtime.h>

#include "vb_common.cuh"
#include "vb_launch.cuh"

namespace vb {

// High word of |v| (sign cleared): orders |v| up to ties of the low word.
__device__ __forceinline__ unsigned hi_key(double v) { return (unsigned)__double2hiint(v) & 0x7fffffffu; }
__device__ __forceinline__ unsigned hi_key(float v) { return __float_as_uint(v) & 0x7fffffffu; }

// Pivot choice of every factor kernel. The key of a candidate row is the top
// 24 bits of |v| (the sign-cleared high word shifted right by 7: the exponent
// and the leading 13 mantissa bits in FP64, 16 in FP32) above 255 - row, so
// one 32-bit max reduction over the warp names the pivot row: the largest
// magnitude to within a relative 2^-13 (FP64) or 2^-16 (FP32), the lowest row
// among those (threshold partial pivoting with threshold 1 - 2^-13; strict
// partial pivoting takes the exact maximum, at the price of a second
// reduction, ballots and shuffles on the pivot chain). A NaN counts as
// magnitude 0. Rows that may not pivot (pivoted, padding) take key 0, below
// every candidate (row <= 127, so a candidate's low byte is >= 128).
template <typename R>
__device__ __forceinline__ unsigned pivot_key32(R v, int row) {
  const unsigned mag = isnan(v) ? 0u : (hi_key(v) >> 7);
  return (mag << 8) | (unsigned)(255 - row);
}
__device__ __forceinline__ int pivot_row(unsigned kmax) { return 255 - (int)(kmax & 255u); }

// Correctly rounded reciprocal (the value of 1 / x).
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }

// Power of two s with s * m in [1, 2) for a finite m > 0 (1 otherwise).
__device__ __forceinline__ double pow2_scale(double m) {
  if (!(m > 0.0) || !isfinite(m)) return 1.0;
  int e;
  frexp(m, &e);               // m = f 2^e, f in [0.5, 1)
  return ldexp(1.0, 1 - e);   // s m = 2 f in [1, 2)
}

// Two values of the factor's element type handed over in one shared-memory access.
template <typename R> struct Pair;
template <> struct Pair<double> { using T = double2; };
template <> struct Pair<float> { using T = float2; };

// ---------------------------------------------------------------- Gauss-Jordan factor
// Shared-memory plan of gj_factor_atmosphere (carved in this order, each
// piece on a 16-byte boundary).
template <int RPL, int CPW, int NW, typename R>
struct GJK {
  static constexpr int NPR = 32 * RPL;          // row capacity (lane l holds rows l + 32 r)
  static constexpr int NPC = CPW * NW;          // column capacity (warp w holds columns w*CPW + c)
  static constexpr int CPWP = (CPW + 1) & ~1;   // stride of a warp's pivot-row slot (pairs)
  __host__ __device__ static size_t al(size_t x) { return (x + 15) & ~(size_t)15; }
  static size_t smem_bytes(int n, int ld, bool dpf, int li = 0, bool pipe = false) {
    const size_t blk = (size_t)n * ld, iblk = (size_t)n * (li ? li : ld);
    return al(iblk * sizeof(R))                       // Ib: the inverse of the layer (natural order, stride li)
           + (dpf ? al(blk * sizeof(double)) : 0)     // Db: the next diagonal block, prefetched
           + al(2 * NPC * sizeof(double))             // rsc: row scales of this and the previous layer (EQ)
           + al(2 * NPR * sizeof(R))                  // colb: multipliers of the next step (2 parities)
           + al(NPR * sizeof(R))                      // rps: 1 / pivot of each row
           + al(4 * NPR * sizeof(double))             // rsb: the next layer's rhs and sub_d rows (2 parities)
           + al((pipe ? 2 : 1) * NW * CPWP * sizeof(R))  // prs: pivot-row hand-over, a slot per warp (x2: parity)
           + al(2 * NPR * sizeof(double))             // vecs: right-hand side ping-pong
           + al(NPC * sizeof(int))                    // pivs: pivot row of each step
           + al(NPR * sizeof(int))                    // qs: step of each pivot row
           + al(2 * sizeof(int))                      // pb: pivot row of the next step (2 parities)
           + 16                                       // mbarrier of the prefetch
           + (pipe ? al(2 * CPW * NPR * sizeof(R))    // colr: multiplier ring, one slot per column of two panels
                         + al(2 * CPW * sizeof(int))  // pring: pivot row of each ring slot
                         + al((2 * CPW + 2) * 8)      // mbarriers: a slot's publication (2 CPW), a panel consumed (2)
                         + 16                         // abort flag
                   : 0);
  }
};

// Factor all layers of one atmosphere by Gauss-Jordan inversion of each
// Schur-updated diagonal block. On entry Din[j] holds D_j (row stride ld); on
// exit out[j] holds A'_j^{-1}; with rhs != nullptr the first sweep of the
// right-hand side rhs[nz][ni] is done in place (solver.py:73-88).
//
// The reference inverts each block by lu_factor then lu_solve(LU, I)
// (solver.py:46-48). Here the inverse comes from one serial chain of ni
// Gauss-Jordan steps instead of three (factor, forward and back
// substitution). Gauss-Jordan bounds the left residual |X B - I| of the
// inverse X of the matrix B it eliminates on. With tr set the elimination
// runs on the transposed block B = A'^T (partial pivoting within a row of
// A'), so X = A'^{-1} has a small right residual |A' X - I| as the
// reference's lu_solve(LU, I) columns do: what solves x = X b need (the Ros2
// step; on the stiff config-0 draw eliminating on A' itself left the block
// solve's normwise backward error at 4e-12 instead of 7e-15). Without tr it
// runs on B = A' (partial pivoting within a column, as lu_factor), for
// callers that solve with X^T (the transposed sweeps of the adjoint), which
// need |X A' - I| small.
//  * Tile in registers: lane l holds rows l + 32 r (r < RPL), warp w columns
//    w*CPW + c (c < CPW) of B. No row exchanges: row p_k is the pivot row
//    of step k. Pivot rows are not normalised during the elimination (row i
//    carries the factor piv_i of its own step), so every element update is
//    one FMA
//        S[i][:] -= m_i S[p][:],   m_i = S[i][k] / piv_k  (m_p = 0),
//    column k becomes -m_i (row p: 1), and each row is scaled by 1/piv_i at
//    the end. The stored result T satisfies B^{-1}[q(i)][p_m] = T[i][m]
//    (q(i): the step whose pivot row is i), applied (transposed back when
//    tr) by the scatter into Ib.
//  * One block barrier per step. During step k the owner warp of column
//    k+1 updates that column first, takes its argmax (one redux.sync on
//    the packed pivot_key32: threshold partial pivoting), inverts the
//    pivot and publishes p_{k+1} with the scaled multipliers; the other warps
//    update meanwhile. A warp takes its part of the pivot row from the owner
//    lane through a per-warp shared slot (no block barrier).
//  * Layer j's Schur update reads Inv_{j-1} from Ib (shared), D_j from Db
//    (bulk-prefetched during layer j-1) when DPF, else from global memory.
//  * EQ (transposed orientation): every row of A'_j is scaled by a power of
//    two bringing its largest magnitude to [1, 2) before the elimination
//    (row equilibration, exact); the stored inverse is X = (R A'_j)^{-1},
//    the scales go to rs_out, and A'_j^{-1} = X diag(r).
//  * li: row stride of Ib and of the stored inverses (ld when 0).
template <int RPL, int CPW, int NW, bool DPF, typename R, bool EQ = false, bool PIPE = false>
__device__ __forceinline__ void gj_factor_atmosphere(int nz, int n, int ld, const double* Din, R* out,
                                                     const double* __restrict__ supn,
                                                     const double* __restrict__ subn, double* rhs,
                                                     bool tr, int32_t* status, char* smem_raw, long long wlim,
                                                     int li = 0, double* rs_out = nullptr,
                                                     long long plim = WAIT_LIMIT) {
  using G = GJK<RPL, CPW, NW, R>;
  using R2 = typename Pair<R>::T;
  constexpr int NPR = G::NPR, CPWP = G::CPWP, NPC = G::NPC;
  if (li == 0) li = ld;
  // value of slot s (warp-uniform) of a per-lane row array
  auto pick = [](const R* v, int s) {
    R x = v[0];
#pragma unroll
    for (int r = 1; r < RPL; ++r) x = (s == r) ? v[r] : x;
    return x;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned FULL = 0xffffffffu;
  const int blk = n * ld, iblk = n * li;
  char* sp = smem_raw;
  auto take = [&](size_t bytes) {
    char* q = sp;
    sp += G::al(bytes);
    return q;
  };
  R* Ib = reinterpret_cast<R*>(take((size_t)iblk * sizeof(R)));
  double* Db = DPF ? reinterpret_cast<double*>(take((size_t)blk * sizeof(double))) : nullptr;
  double* rsc = reinterpret_cast<double*>(take(2 * NPC * sizeof(double)));
  R* colb = reinterpret_cast<R*>(take(2 * NPR * sizeof(R)));
  R* rps = reinterpret_cast<R*>(take(NPR * sizeof(R)));
  double* rsb = reinterpret_cast<double*>(take(4 * NPR * sizeof(double)));
  R* prs = reinterpret_cast<R*>(take((PIPE ? 2 : 1) * NW * G::CPWP * sizeof(R)));
  double* vecs = reinterpret_cast<double*>(take(2 * NPR * sizeof(double)));
  int* pivs = reinterpret_cast<int*>(take(G::NPC * sizeof(int)));
  int* qs = reinterpret_cast<int*>(take(NPR * sizeof(int)));
  int* pb = reinterpret_cast<int*>(take(2 * sizeof(int)));
  uint64_t* bar = reinterpret_cast<uint64_t*>(take(16));
  R* colr = PIPE ? reinterpret_cast<R*>(take(2 * CPW * NPR * sizeof(R))) : nullptr;
  int* pring = PIPE ? reinterpret_cast<int*>(take(2 * CPW * sizeof(int))) : nullptr;
  uint64_t* fbar = PIPE ? reinterpret_cast<uint64_t*>(take((2 * CPW + 2) * 8)) : nullptr;
  uint64_t* ebar = PIPE ? fbar + 2 * CPW : nullptr;
  volatile int* abortp = PIPE ? reinterpret_cast<volatile int*>(take(16)) : nullptr;
  const uint32_t dbytes = (uint32_t)(blk * sizeof(double));
  int st_local = 0;
  // pipeline signals: fbar[s] completes when the owner warp of ring slot s
  // has published it (32 arrivals), ebar[x] when every warp has applied a
  // panel of parity x (32 NW arrivals)
  auto pipe_init = [&]() {
#pragma unroll 1
    for (int s2 = 0; s2 < 2 * CPW; ++s2) mbar_init(fbar + s2, 32);
    mbar_init(ebar, 32 * NW);
    mbar_init(ebar + 1, 32 * NW);
  };

  for (int e = threadIdx.x; e < iblk; e += blockDim.x) Ib[e] = R(0);   // the padding columns stay 0
  if (rhs)
    for (int i = threadIdx.x; i < n; i += blockDim.x) vecs[i] = rhs[i];
  if (DPF && threadIdx.x == 0) mbar_init(bar, 1);
  if (PIPE && threadIdx.x == 0) {
    pipe_init();
    *abortp = 0;
  }
  __syncthreads();
  if (DPF && threadIdx.x == 0) {
    mbar_expect_tx(bar, dbytes);
    bulk_g2s(Db, Din, dbytes, bar);
  }

  // argmax of column kn (values t, already updated) over the unpivoted rows,
  // run by the warp that owns the column (pivot_key32: one max reduction
  // names the row); the pivot value comes from its owner lane.
  auto pivot_of = [&](const R (&t)[RPL], unsigned used, R& piv) {
    unsigned km = 0u;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int i = lane + 32 * r;
      if (i < n && !((used >> r) & 1u)) km = max(km, pivot_key32(t[r], i));
    }
    const int p1 = pivot_row(__reduce_max_sync(FULL, km));
    piv = __shfl_sync(FULL, pick(t, p1 >> 5), p1 & 31);
    return p1;
  };
  // multipliers t / piv of step kn into cb (0 on the pivot row), its pivot
  // row into *pbp, pivs[kn], qs[p1] and 1 / piv into rps[p1]
  auto store_step_rp = [&](const R (&t)[RPL], int p1, R piv, R rp, int kn, R* cb, int* pbp, R (&mo)[RPL]) {
    if (piv == R(0)) st_local |= VB_STATUS_ZERO_PIVOT;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int i = lane + 32 * r;
      mo[r] = (i < n && i != p1) ? t[r] * rp : R(0);
      cb[i] = mo[r];
    }
    *pbp = p1;   // every lane stores the same values
    pivs[kn] = p1;
    qs[p1] = kn;
    rps[p1] = rp;
  };
  auto store_step = [&](const R (&t)[RPL], int p1, R piv, int kn, R* cb, int* pbp, R (&mo)[RPL]) {
    store_step_rp(t, p1, piv, rcp_rn(piv), kn, cb, pbp, mo);
  };
  auto publish = [&](const R (&t)[RPL], unsigned used, int kn, R* cb, int* pbp, R (&mo)[RPL]) {
    R piv;
    const int p1 = pivot_of(t, used, piv);
    store_step(t, p1, piv, kn, cb, pbp, mo);
    return p1;
  };

  R a[RPL][CPW];

  // PIPE: the same elimination without a block barrier per step. The warp
  // that owns column k publishes step k (pivot row, multipliers) into ring
  // slot (panel parity, column in panel) and signals fbar of the slot; the
  // owner of a panel runs its steps back to back from registers while the
  // other warps apply the published steps as they arrive. Before a panel
  // reuses the slots of the panel two before it, its owner waits until every
  // warp has applied that panel (ebar). Panel numbers and barrier phases
  // restart every layer (a partial last panel publishes fewer slots). Every
  // wait is bounded; a warp that gives up raises *abortp, which ends every
  // other wait, and the layer's caller reports VB_STATUS_WATCHDOG.
  auto eliminate_pipelined = [&](unsigned& used) {
    bool dead = false;
    auto fail = [&](bool ok) {
      if (__any_sync(FULL, !ok)) {
        dead = true;
        *abortp = 1;
      }
    };
    // multipliers, pivot row and this warp's part of the pivot row of the
    // step this warp published last: the owner of a panel runs its steps
    // from these registers. The publisher takes its part of the pivot row
    // by shuffles as soon as the argmax has named the row, while the
    // reciprocal is in flight and before the other warps wake.
    R mk[RPL], pn[CPW];
    int pk = 0;
    // Publishing step kn from column values t: the argmax, then this warp's
    // part of the new pivot row pk into pn (through the warp's hand-over slot
    // of step kn's parity), then the multipliers and the signal.
    auto fetch_row = [&](int kn) {
      R* ph = prs + ((kn & 1) * NW + warp) * CPWP;
      const int ps = pk >> 5, po = pk & 31;
#pragma unroll
      for (int r = 0; r < RPL; ++r)
        if (r == ps && lane == po) {
#pragma unroll
          for (int c2 = 0; c2 < CPWP; c2 += 2)
            reinterpret_cast<R2*>(ph)[c2 / 2] = R2{a[r][c2], c2 + 1 < CPW ? a[r][c2 + 1] : R(0)};
        }
      __syncwarp();
#pragma unroll
      for (int c2 = 0; c2 < CPW; c2 += 2) {
        const R2 v = reinterpret_cast<const R2*>(ph)[c2 / 2];
        pn[c2] = v.x;
        if (c2 + 1 < CPW) pn[c2 + 1] = v.y;
      }
    };
    if (warp == 0) {
      R t[RPL], piv;
#pragma unroll
      for (int r = 0; r < RPL; ++r) t[r] = a[r][0];
      pk = pivot_of(t, 0u, piv);
      fetch_row(0);
      store_step(t, pk, piv, 0, colr, pring, mk);
      mbar_arrive(fbar);
    }
#pragma unroll 1
    for (int w0 = 0; w0 < NW; ++w0) {
      if (w0 * CPW >= n || dead) break;
#pragma unroll
      for (int c = 0; c < CPW; ++c) {
        const int k = w0 * CPW + c;
        if (k < n && !dead) {
          R t[RPL];          // column k+1 after this step, when this warp publishes step k+1
          bool pub = false;  // (warp-uniform)
          int sn = 0;        // and its ring slot
          if (warp == w0) {
            // ---- owner of column k: the step from registers (pn: its part
            //      of the pivot row, taken when the step was published)
            const int p = pk, ps = p >> 5, po = p & 31;
            R m[RPL];
#pragma unroll
            for (int r = 0; r < RPL; ++r) {
              m[r] = mk[r];
              if (r == ps && lane == po) used |= 1u << r;
            }
            pub = c + 1 < CPW && k + 1 < n;   // column k+1 is this warp's too
            sn = (w0 & 1) * CPW + (c + 1) % CPW;
#pragma unroll
            for (int r = 0; r < RPL; ++r) t[r] = fma(-m[r], pn[(c + 1) % CPW], a[r][(c + 1) % CPW]);
#pragma unroll
            for (int r = 0; r < RPL; ++r)
#pragma unroll
              for (int c2 = 0; c2 < CPW; ++c2) a[r][c2] = fma(-m[r], pn[c2], a[r][c2]);
#pragma unroll
            for (int r = 0; r < RPL; ++r) a[r][c] = (lane + 32 * r == p) ? R(1) : -m[r];
          } else {
            // ---- every other warp: wait for the slot, then the step from
            //      shared memory (pivot row through a per-warp hand-over slot,
            //      two by step parity: one __syncwarp per step)
            const int sl = (w0 & 1) * CPW + c;
            fail(mbar_wait_or_abort(fbar + sl, (uint32_t)((w0 >> 1) & 1), plim, abortp));
            if (!dead) {
              const int p = pring[sl], ps = p >> 5, po = p & 31;
              R m[RPL];
#pragma unroll
              for (int r = 0; r < RPL; ++r) {
                m[r] = colr[sl * NPR + lane + 32 * r];
                if (r == ps && lane == po) used |= 1u << r;
              }
              R* ph = prs + ((k & 1) * NW + warp) * CPWP;
#pragma unroll
              for (int r = 0; r < RPL; ++r)
                if (r == ps && lane == po) {
#pragma unroll
                  for (int c2 = 0; c2 < CPWP; c2 += 2)
                    reinterpret_cast<R2*>(ph)[c2 / 2] = R2{a[r][c2], c2 + 1 < CPW ? a[r][c2 + 1] : R(0)};
                }
              __syncwarp();
              R prow[CPWP];
#pragma unroll
              for (int c2 = 0; c2 < CPWP; c2 += 2) {
                const R2 v = reinterpret_cast<const R2*>(ph)[c2 / 2];
                prow[c2] = v.x;
                prow[c2 + 1] = v.y;
              }
              // column k+1 opens this warp's panel: it publishes step k+1
              pub = c + 1 == CPW && k + 1 < n && warp == w0 + 1;
#pragma unroll
              for (int r = 0; r < RPL; ++r) t[r] = fma(-m[r], prow[0], a[r][0]);
#pragma unroll
              for (int r = 0; r < RPL; ++r)
#pragma unroll
                for (int c2 = 0; c2 < CPW; ++c2) a[r][c2] = fma(-m[r], prow[c2], a[r][c2]);
              if (pub) {
                // into the slots of the panel two before, once every warp has applied it
                const int pnl = w0 + 1;
                sn = (pnl & 1) * CPW;
                if (pnl >= 2)
                  fail(mbar_wait_or_abort(ebar + (pnl & 1), (uint32_t)(((pnl - 2) >> 1) & 1), plim, abortp));
              }
            }
          }
          if (pub && !dead) {
            R piv;
            pk = pivot_of(t, used, piv);
            fetch_row(k + 1);
            store_step(t, pk, piv, k + 1, colr + sn * NPR, pring + sn, mk);
            mbar_arrive(fbar + sn);
          }
          if (!dead && (c + 1 == CPW || k + 1 == n)) mbar_arrive(ebar + (w0 & 1));   // panel w0 applied
        }
      }
    }
  };

  for (int j = 0; j < nz; ++j) {
    if (DPF) {
      const bool ok = mbar_wait(bar, (uint32_t)(j & 1), wlim);
      if (__syncthreads_or(!ok)) {
        // give up: wait (bounded) for the copy still in flight, report, return
        if (threadIdx.x == 0) {
          mbar_wait(bar, (uint32_t)(j & 1), WAIT_LIMIT);
          atomicOr(status, VB_STATUS_WATCHDOG);
        }
        return;
      }
    }
    // the next layer's rhs and sub_d rows, for the forward sweep at the end of the layer
    double rn = 0.0, sn = 0.0;
    const bool ride = rhs && j + 1 < nz && (int)threadIdx.x < n;
    if (ride) {
      rn = rhs[(int64_t)(j + 1) * n + threadIdx.x];
      sn = subn[(int64_t)j * n + threadIdx.x];
    }
    // ---- D_j and the Hadamard Schur update from Inv_{j-1} (solver.py:47):
    //      tile element (i, m) = B[i][m], A'_j[m][i] when tr, else A'_j[i][m]
    {
      const double* D = DPF ? Db : Din + (int64_t)j * blk;
      double sr[RPL], sc[CPW];   // the sub_d / sup_d factor of tile row i and column m
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        sr[r] = (j > 0 && i < n) ? (tr ? supn : subn)[(int64_t)(j - 1) * n + i] : 0.0;
      }
#pragma unroll
      for (int c = 0; c < CPW; ++c) {
        const int m = warp * CPW + c;
        sc[c] = (j > 0 && m < n) ? (tr ? subn : supn)[(int64_t)(j - 1) * n + m] : 0.0;
      }
      const int si = tr ? 1 : ld, sm = tr ? ld : 1;   // element strides of tile rows / columns in D
      const int ii = tr ? 1 : li, im = tr ? li : 1;   // and in Ib
      const double* rprev = rsc + ((j + 1) & 1) * NPC;
      double v[RPL][CPW];
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
#pragma unroll
        for (int c = 0; c < CPW; ++c) {
          const int m = warp * CPW + c;
          double x = 0.0;
          if (i < n && m < n) {
            x = D[i * si + m * sm];
            if (j > 0) {
              const double cb = tr ? sc[c] * sr[r] : sr[r] * sc[c];
              double inv = (double)Ib[i * ii + m * im];
              if (EQ) inv = inv * rprev[i];
              x = x - cb * inv;
            }
          }
          v[r][c] = x;
        }
      }
      if (EQ) {
        // largest magnitude of each tile column (row m of A'_j): the column lives in this warp
        double* rcur = rsc + (j & 1) * NPC;
#pragma unroll
        for (int c = 0; c < CPW; ++c) {
          double cm = 0.0;
#pragma unroll
          for (int r = 0; r < RPL; ++r) cm = fmax(cm, fabs(v[r][c]));
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) cm = fmax(cm, __shfl_xor_sync(FULL, cm, off));
          const double s = pow2_scale(cm);
          const int m = warp * CPW + c;
          if (lane == 0 && m < n) {
            rcur[m] = s;
            rs_out[(int64_t)j * n + m] = s;
          }
#pragma unroll
          for (int r = 0; r < RPL; ++r) v[r][c] *= s;
        }
      }
#pragma unroll
      for (int r = 0; r < RPL; ++r)
#pragma unroll
        for (int c = 0; c < CPW; ++c) a[r][c] = (R)v[r][c];
    }
    double* rsj = rsb + (j & 1) * 2 * NPR;   // read by this layer's forward sweep
    if (ride) {
      rsj[threadIdx.x] = rn;
      rsj[NPR + threadIdx.x] = sn;
    }
    __syncthreads();   // Db and Ib consumed
    if (DPF && threadIdx.x == 0 && j + 1 < nz) {
      fence_proxy_async();
      mbar_expect_tx(bar, dbytes);
      bulk_g2s(Db, Din + (int64_t)(j + 1) * blk, dbytes, bar);
    }
    unsigned used = 0;   // rows lane + 32 r already pivoted
    if constexpr (PIPE) {
      eliminate_pipelined(used);
      __syncthreads();
      if (*abortp) {
        // a wait gave up: drain the prefetch in flight, report, return
        if (threadIdx.x == 0) {
          if (DPF && j + 1 < nz) mbar_wait(bar, (uint32_t)((j + 1) & 1), WAIT_LIMIT);
          atomicOr(status, VB_STATUS_WATCHDOG);
        }
        return;
      }
      if (threadIdx.x == 0) {   // every signal of this layer has completed: restart the phases
#pragma unroll 1
        for (int s2 = 0; s2 < 2 * CPW + 2; ++s2) mbar_inval(fbar + s2);
        pipe_init();
      }
    } else {
    // the warp that published a step applies it from its registers (the
    // owner of column k published step k: no shared-memory round trip on
    // the lookahead warp's path in five of six steps)
    R mo[RPL];
    int pk = 0;
    if (warp == 0) {
      R t[RPL];
#pragma unroll
      for (int r = 0; r < RPL; ++r) t[r] = a[r][0];
      pk = publish(t, 0u, 0, colb, pb, mo);
    }
    __syncthreads();
    // ================================================================ elimination
#pragma unroll 1
    for (int w0 = 0; w0 < NW; ++w0) {
      if (w0 * CPW >= n) break;
#pragma unroll
      for (int c = 0; c < CPW; ++c) {
        const int k = w0 * CPW + c;
        if (k < n) {
          int p;
          R m[RPL];
          if (warp == w0) {
            p = pk;
#pragma unroll
            for (int r = 0; r < RPL; ++r) m[r] = mo[r];
          } else {
            p = pb[k & 1];
#pragma unroll
            for (int r = 0; r < RPL; ++r) m[r] = colb[(k & 1) * NPR + lane + 32 * r];
          }
          const int ps = p >> 5, po = p & 31;
#pragma unroll
          for (int r = 0; r < RPL; ++r)
            if (r == ps && lane == po) used |= 1u << r;
          // this warp's part of the pivot row, from its owner lane (pair
          // stores predicated on the slot: no selects)
          R* ph = prs + warp * CPWP;
#pragma unroll
          for (int r = 0; r < RPL; ++r)
            if (r == ps && lane == po) {
#pragma unroll
              for (int c2 = 0; c2 < CPWP; c2 += 2)
                reinterpret_cast<R2*>(ph)[c2 / 2] = R2{a[r][c2], c2 + 1 < CPW ? a[r][c2 + 1] : R(0)};
            }
          __syncwarp();
          R prow[CPWP];
#pragma unroll
          for (int c2 = 0; c2 < CPWP; c2 += 2) {
            const R2 v = reinterpret_cast<const R2*>(ph)[c2 / 2];
            prow[c2] = v.x;
            prow[c2 + 1] = v.y;
          }
          const int cl = (c + 1) % CPW;                     // column k+1: slot and owner warp
          const int wl = (c + 1 < CPW) ? w0 : w0 + 1;
          if (k + 1 < n && warp == wl) {
            R t[RPL], piv;
#pragma unroll
            for (int r = 0; r < RPL; ++r) t[r] = fma(-m[r], prow[cl], a[r][cl]);
            const int p1 = pivot_of(t, used, piv);
            const R rp = rcp_rn(piv);   // in flight while the rest of step k is applied
#pragma unroll
            for (int r = 0; r < RPL; ++r)
#pragma unroll
              for (int c2 = 0; c2 < CPW; ++c2) a[r][c2] = fma(-m[r], prow[c2], a[r][c2]);
            store_step_rp(t, p1, piv, rp, k + 1, colb + ((k + 1) & 1) * NPR, pb + ((k + 1) & 1), mo);
            pk = p1;
          } else {
#pragma unroll
            for (int r = 0; r < RPL; ++r)
#pragma unroll
              for (int c2 = 0; c2 < CPW; ++c2) a[r][c2] = fma(-m[r], prow[c2], a[r][c2]);
          }
          if (warp == w0) {
#pragma unroll
            for (int r = 0; r < RPL; ++r) a[r][c] = (lane + 32 * r == p) ? R(1) : -m[r];
          }
          __syncthreads();
        }
      }
    }
    }
    // ---- scale rows by 1/piv, scatter B^{-1}[q(i)][p_m] = T[i][m] into Ib
    //      (A'^{-1}[p_m][q(i)] when tr; q(i) = qs[i], the step pivoting on row i)
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int i = lane + 32 * r;
      if (i < n) {
        const R s = rps[i];
        const int qi = qs[i];
#pragma unroll
        for (int c = 0; c < CPW; ++c) {
          const int m = warp * CPW + c;
          if (m < n) {
            const R v = a[r][c] * s;
            if (!isfinite(v)) st_local |= VB_STATUS_NONFINITE;
            Ib[tr ? pivs[m] * li + qi : qi * li + pivs[m]] = v;
          }
        }
      }
    }
    __syncthreads();
    // ---- Inv_j to global memory (natural order, padding columns 0)
    {
      R2* O = reinterpret_cast<R2*>(out + (int64_t)j * iblk);
      const R2* S2 = reinterpret_cast<const R2*>(Ib);
      for (int e = threadIdx.x; e < iblk / 2; e += blockDim.x) O[e] = S2[e];
    }
    // ---- forward sweep of the right-hand side: rhs[j+1] -= sub_d[j] o (Inv_j rhs[j])
    if (rhs && j + 1 < nz) {
      const double* vc = vecs + (j & 1) * NPR;
      double* vn = vecs + ((j + 1) & 1) * NPR;
      // four lanes per row, eight rows per warp per pass (warp-uniform passes)
      const int sub = lane & 3;
      for (int i0 = warp * 8; i0 < n; i0 += NW * 8) {
        const int i = i0 + (lane >> 2);
        double s0 = 0.0, s1 = 0.0;
        if (i < n) {
          int m = sub;
          for (; m + 4 < n; m += 8) {
            s0 = fma((double)Ib[i * li + m], vc[m], s0);
            s1 = fma((double)Ib[i * li + m + 4], vc[m + 4], s1);
          }
          if (m < n) s0 = fma((double)Ib[i * li + m], vc[m], s0);
        }
        double s = s0 + s1;
        s += __shfl_xor_sync(FULL, s, 1);
        s += __shfl_xor_sync(FULL, s, 2);
        if (sub == 0 && i < n) {
          const double v = rsj[i] - rsj[NPR + i] * s;
          rhs[(int64_t)(j + 1) * n + i] = v;
          vn[i] = v;
        }
      }
    }
  }
  if (st_local) atomicOr(status, st_local);
}

// ---------------------------------------------------------------- paired Gauss-Jordan factor
// Two atmospheres of one uniform batch per CTA, their pivot chains
// interleaved in the same warps: every warp holds both atmospheres' tiles
// (the single kernel's layout), each step's loads, hand-overs and updates are
// issued for both, and the warp owning the next column takes both argmaxes
// and reciprocals back to back, so the two chains' latencies overlap and one
// block barrier serves both. The arithmetic of each atmosphere is the single
// kernel's, in the same order (FP64, transposed orientation when tr).

// Row-slot value of a per-lane row array (s warp-uniform).
template <int RPL>
__device__ __forceinline__ double pick_slot(const double (&v)[RPL], int s) {
  double x = v[0];
#pragma unroll
  for (int r = 1; r < RPL; ++r) x = (s == r) ? v[r] : x;
  return x;
}

// Argmaxes of two columns (one per atmosphere), interleaved: both keys
// (pivot_key32) reduced back to back, then both pivot values shuffled from
// their owner lanes. The chosen rows equal the single kernel's.
template <int RPL>
__device__ __forceinline__ void pivot_pair(const double (&t)[2][RPL], const unsigned (&used)[2], int n,
                                           int (&p1)[2], double (&piv)[2]) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  unsigned km[2] = {0u, 0u};
#pragma unroll
  for (int e = 0; e < 2; ++e)
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int i = lane + 32 * r;
      if (i < n && !((used[e] >> r) & 1u)) km[e] = max(km[e], pivot_key32(t[e][r], i));
    }
  const unsigned m1a = __reduce_max_sync(FULL, km[0]);
  const unsigned m1b = __reduce_max_sync(FULL, km[1]);
  p1[0] = pivot_row(m1a);
  p1[1] = pivot_row(m1b);
  piv[0] = __shfl_sync(FULL, pick_slot(t[0], p1[0] >> 5), p1[0] & 31);
  piv[1] = __shfl_sync(FULL, pick_slot(t[1], p1[1] >> 5), p1[1] & 31);
}

// Shared-memory plan of the paired factor: per atmosphere (carved in this
// order, each piece on a 16-byte boundary) the inverse of the layer, the
// prefetched next block, multipliers (2 parities), 1/pivot per row, the next
// layer's rhs and sub_d rows (2 parities), the per-warp pivot-row hand-over,
// the rhs ping-pong, pivot row per step, step per pivot row, the next
// step's pivot row (2 parities) and the prefetch mbarrier.
template <int RPL, int CPW, int NW>
struct GJP {
  static constexpr int NPR = 32 * RPL, NPC = CPW * NW, CPWP = (CPW + 1) & ~1;
  __host__ __device__ static size_t al(size_t x) { return (x + 15) & ~(size_t)15; }
  static size_t one_bytes(int n, int ld) {
    const size_t blk = (size_t)n * ld * sizeof(double);
    return 2 * al(blk) + al(2 * NPR * 8) + al(NPR * 8) + al(4 * NPR * 8) + al(NW * CPWP * 8) + al(2 * NPR * 8) +
           al(NPC * 4) + al(NPR * 4) + al(2 * 4) + 16;
  }
  static size_t smem_bytes(int n, int ld) { return 2 * one_bytes(n, ld); }
};

struct PairPtrs {
  const double* Din[2];  // D_j of each atmosphere (row stride ld), layer-major
  double* out[2];        // inverses (may equal Din: in place)
  const double* supn[2];
  const double* subn[2];
  double* rhs[2];        // rhs rows for the ride-along forward sweep, or nullptr
  int32_t* status[2];
};

// Publishes step KN of both atmospheres from their column values T (the
// single kernel's store of the multipliers, pivot rows and reciprocals, into
// parity PAR); written as a macro so the register arrays it updates never
// leave registers.
#define VB_PAIR_PUBLISH(T, KN, PAR)                                            \
  do {                                                                         \
    int p1_[2];                                                                \
    double piv_[2], rp_[2];                                                    \
    pivot_pair<RPL>(T, used, n, p1_, piv_);                                    \
    _Pragma("unroll") for (int e_ = 0; e_ < 2; ++e_) {                         \
      if (piv_[e_] == 0.0) st_local[e_] |= VB_STATUS_ZERO_PIVOT;               \
      rp_[e_] = rcp_rn(piv_[e_]);                                              \
    }                                                                          \
    _Pragma("unroll") for (int e_ = 0; e_ < 2; ++e_) {                         \
      _Pragma("unroll") for (int r_ = 0; r_ < RPL; ++r_) {                     \
        const int i_ = lane + 32 * r_;                                         \
        mo[e_][r_] = (i_ < n && i_ != p1_[e_]) ? T[e_][r_] * rp_[e_] : 0.0;    \
        colb[e_][(PAR) * NPR + i_] = mo[e_][r_];                               \
      }                                                                        \
      pb[e_][PAR] = p1_[e_];                                                   \
      pivs[e_][KN] = p1_[e_];                                                  \
      qs[e_][p1_[e_]] = (KN);                                                  \
      rps[e_][p1_[e_]] = rp_[e_];                                              \
      pk[e_] = p1_[e_];                                                        \
    }                                                                          \
  } while (0)

template <int RPL, int CPW, int NW>
__device__ __forceinline__ void gj_factor_pair(int nz, int n, int ld, const PairPtrs& P, bool tr, char* smem_raw,
                                               long long wlim) {
  using G = GJP<RPL, CPW, NW>;
  constexpr int NPR = G::NPR, CPWP = G::CPWP;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned FULL = 0xffffffffu;
  const int blk = n * ld;
  const bool with_rhs = P.rhs[0] != nullptr;
  double *Ib[2], *Db[2], *colb[2], *rps[2], *rsb[2], *prs[2], *vecs[2];
  int *pivs[2], *qs[2], *pb[2];
  uint64_t* bar[2];
  {
    char* sp = smem_raw;
    auto take = [&](size_t bytes) {
      char* q = sp;
      sp += G::al(bytes);
      return q;
    };
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      Ib[e] = reinterpret_cast<double*>(take((size_t)blk * 8));
      Db[e] = reinterpret_cast<double*>(take((size_t)blk * 8));
      colb[e] = reinterpret_cast<double*>(take(2 * NPR * 8));
      rps[e] = reinterpret_cast<double*>(take(NPR * 8));
      rsb[e] = reinterpret_cast<double*>(take(4 * NPR * 8));
      prs[e] = reinterpret_cast<double*>(take(NW * CPWP * 8));
      vecs[e] = reinterpret_cast<double*>(take(2 * NPR * 8));
      pivs[e] = reinterpret_cast<int*>(take(G::NPC * 4));
      qs[e] = reinterpret_cast<int*>(take(NPR * 4));
      pb[e] = reinterpret_cast<int*>(take(2 * 4));
      bar[e] = reinterpret_cast<uint64_t*>(take(16));
    }
  }
  const uint32_t dbytes = (uint32_t)(blk * sizeof(double));
  int st_local[2] = {0, 0};
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    for (int q = threadIdx.x; q < blk; q += blockDim.x) Ib[e][q] = 0.0;   // the padding columns stay 0
    if (with_rhs)
      for (int i = threadIdx.x; i < n; i += blockDim.x) vecs[e][i] = P.rhs[e][i];
  }
  if (threadIdx.x == 0) {
    mbar_init(bar[0], 1);
    mbar_init(bar[1], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      mbar_expect_tx(bar[e], dbytes);
      bulk_g2s(Db[e], P.Din[e], dbytes, bar[e]);
    }
  }
  double a[2][RPL][CPW];
  for (int j = 0; j < nz; ++j) {
    {
      const bool ok0 = mbar_wait(bar[0], (uint32_t)(j & 1), wlim);
      const bool ok1 = mbar_wait(bar[1], (uint32_t)(j & 1), wlim);
      if (__syncthreads_or(!(ok0 && ok1))) {
        // give up: wait (bounded) for the copies still in flight, report, return
        if (threadIdx.x == 0) {
          mbar_wait(bar[0], (uint32_t)(j & 1), WAIT_LIMIT);
          mbar_wait(bar[1], (uint32_t)(j & 1), WAIT_LIMIT);
          atomicOr(P.status[0], VB_STATUS_WATCHDOG);
          atomicOr(P.status[1], VB_STATUS_WATCHDOG);
        }
        return;
      }
    }
    // the next layer's rhs and sub_d rows, for the forward sweeps at the end of the layer
    double rn[2] = {0.0, 0.0}, sn[2] = {0.0, 0.0};
    const bool ride = with_rhs && j + 1 < nz && (int)threadIdx.x < n;
    if (ride) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        rn[e] = P.rhs[e][(int64_t)(j + 1) * n + threadIdx.x];
        sn[e] = P.subn[e][(int64_t)j * n + threadIdx.x];
      }
    }
    // ---- D_j and the Hadamard Schur update from Inv_{j-1} (solver.py:47)
    {
      const int si = tr ? 1 : ld, sm = tr ? ld : 1;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        double sr[RPL], sc[CPW];
#pragma unroll
        for (int r = 0; r < RPL; ++r) {
          const int i = lane + 32 * r;
          sr[r] = (j > 0 && i < n) ? (tr ? P.supn[e] : P.subn[e])[(int64_t)(j - 1) * n + i] : 0.0;
        }
#pragma unroll
        for (int c = 0; c < CPW; ++c) {
          const int m = warp * CPW + c;
          sc[c] = (j > 0 && m < n) ? (tr ? P.subn[e] : P.supn[e])[(int64_t)(j - 1) * n + m] : 0.0;
        }
#pragma unroll
        for (int r = 0; r < RPL; ++r) {
          const int i = lane + 32 * r;
#pragma unroll
          for (int c = 0; c < CPW; ++c) {
            const int m = warp * CPW + c;
            double x = 0.0;
            if (i < n && m < n) {
              x = Db[e][i * si + m * sm];
              if (j > 0) {
                const double cb = tr ? sc[c] * sr[r] : sr[r] * sc[c];
                double inv = Ib[e][i * si + m * sm];
                x = x - cb * inv;
              }
            }
            a[e][r][c] = x;
          }
        }
        double* rsj = rsb[e] + (j & 1) * 2 * NPR;   // read by this layer's forward sweep
        if (ride) {
          rsj[threadIdx.x] = rn[e];
          rsj[NPR + threadIdx.x] = sn[e];
        }
      }
    }
    __syncthreads();   // Db and Ib consumed
    if (threadIdx.x == 0 && j + 1 < nz) {
      fence_proxy_async();
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        mbar_expect_tx(bar[e], dbytes);
        bulk_g2s(Db[e], P.Din[e] + (int64_t)(j + 1) * blk, dbytes, bar[e]);
      }
    }
    // ================================================================ elimination (both chains)
    unsigned used[2] = {0u, 0u};   // rows lane + 32 r already pivoted
    double mo[2][RPL];             // multipliers of the step this warp published
    int pk[2] = {0, 0};            // and its pivot rows
    if (warp == 0) {
      double t[2][RPL];
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int r = 0; r < RPL; ++r) t[e][r] = a[e][r][0];
      VB_PAIR_PUBLISH(t, 0, 0);
    }
    __syncthreads();
#pragma unroll 1
    for (int w0 = 0; w0 < NW; ++w0) {
      if (w0 * CPW >= n) break;
#pragma unroll
      for (int c = 0; c < CPW; ++c) {
        const int k = w0 * CPW + c;
        if (k < n) {
          int p[2];
          double m[2][RPL];
          if (warp == w0) {   // this warp published step k: from its registers
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              p[e] = pk[e];
#pragma unroll
              for (int r = 0; r < RPL; ++r) m[e][r] = mo[e][r];
            }
          } else {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              p[e] = pb[e][k & 1];
#pragma unroll
              for (int r = 0; r < RPL; ++r) m[e][r] = colb[e][(k & 1) * NPR + lane + 32 * r];
            }
          }
          // this warp's parts of both pivot rows, from their owner lanes
          double prow[2][CPWP];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int ps = p[e] >> 5, po = p[e] & 31;
            double* ph = prs[e] + warp * CPWP;
#pragma unroll
            for (int r = 0; r < RPL; ++r)
              if (r == ps && lane == po) {
                used[e] |= 1u << r;
#pragma unroll
                for (int c2 = 0; c2 < CPWP; c2 += 2)
                  reinterpret_cast<double2*>(ph)[c2 / 2] =
                      make_double2(a[e][r][c2], c2 + 1 < CPW ? a[e][r][c2 + 1] : 0.0);
              }
          }
          __syncwarp();
#pragma unroll
          for (int e = 0; e < 2; ++e)
#pragma unroll
            for (int c2 = 0; c2 < CPWP; c2 += 2) {
              const double2 v = reinterpret_cast<const double2*>(prs[e] + warp * CPWP)[c2 / 2];
              prow[e][c2] = v.x;
              prow[e][c2 + 1] = v.y;
            }
          const int cl = (c + 1) % CPW;   // column k+1: slot and owner warp
          const int wl = (c + 1 < CPW) ? w0 : w0 + 1;
          if (k + 1 < n && warp == wl) {
            double t[2][RPL];
#pragma unroll
            for (int e = 0; e < 2; ++e)
#pragma unroll
              for (int r = 0; r < RPL; ++r) t[e][r] = fma(-m[e][r], prow[e][cl], a[e][r][cl]);
            VB_PAIR_PUBLISH(t, k + 1, (k + 1) & 1);
          }
#pragma unroll
          for (int e = 0; e < 2; ++e)
#pragma unroll
            for (int r = 0; r < RPL; ++r)
#pragma unroll
              for (int c2 = 0; c2 < CPW; ++c2) a[e][r][c2] = fma(-m[e][r], prow[e][c2], a[e][r][c2]);
          if (warp == w0) {
#pragma unroll
            for (int e = 0; e < 2; ++e)
#pragma unroll
              for (int r = 0; r < RPL; ++r) a[e][r][c] = (lane + 32 * r == p[e]) ? 1.0 : -m[e][r];
          }
          __syncthreads();
        }
      }
    }
    // ---- scale rows by 1/piv, scatter B^{-1}[q(i)][p_m] = T[i][m] into Ib
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        if (i < n) {
          const double s = rps[e][i];
          const int qi = qs[e][i];
#pragma unroll
          for (int c = 0; c < CPW; ++c) {
            const int m = warp * CPW + c;
            if (m < n) {
              const double v = a[e][r][c] * s;
              if (!isfinite(v)) st_local[e] |= VB_STATUS_NONFINITE;
              Ib[e][tr ? pivs[e][m] * ld + qi : qi * ld + pivs[e][m]] = v;
            }
          }
        }
      }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      // ---- Inv_j to global memory (natural order, padding columns 0)
      double2* O = reinterpret_cast<double2*>(P.out[e] + (int64_t)j * blk);
      const double2* S2 = reinterpret_cast<const double2*>(Ib[e]);
      for (int q = threadIdx.x; q < blk / 2; q += blockDim.x) O[q] = S2[q];
      // ---- forward sweep of the right-hand side: rhs[j+1] -= sub_d[j] o (Inv_j rhs[j])
      if (with_rhs && j + 1 < nz) {
        const double* vc = vecs[e] + (j & 1) * NPR;
        double* vn = vecs[e] + ((j + 1) & 1) * NPR;
        const double* rsj = rsb[e] + (j & 1) * 2 * NPR;
        const int sub = lane & 3;   // four lanes per row, eight rows per warp per pass
        for (int i0 = warp * 8; i0 < n; i0 += NW * 8) {
          const int i = i0 + (lane >> 2);
          double s0 = 0.0, s1 = 0.0;
          if (i < n) {
            int m = sub;
            for (; m + 4 < n; m += 8) {
              s0 = fma(Ib[e][i * ld + m], vc[m], s0);
              s1 = fma(Ib[e][i * ld + m + 4], vc[m + 4], s1);
            }
            if (m < n) s0 = fma(Ib[e][i * ld + m], vc[m], s0);
          }
          double s = s0 + s1;
          s += __shfl_xor_sync(FULL, s, 1);
          s += __shfl_xor_sync(FULL, s, 2);
          if (sub == 0 && i < n) {
            const double v = rsj[i] - rsj[NPR + i] * s;
            P.rhs[e][(int64_t)(j + 1) * n + i] = v;
            vn[i] = v;
          }
        }
      }
    }
  }
#pragma unroll
  for (int e = 0; e < 2; ++e)
    if (st_local[e]) atomicOr(P.status[e], st_local[e]);
}
#undef VB_PAIR_PUBLISH

// Two atmospheres per CTA (2 blockIdx.x, 2 blockIdx.x + 1) of a uniform
// batch; the inverses replace the blocks in the workspace.
template <int RPL, int CPW, int NW>
__global__ void __launch_bounds__(NW * 32, 1)
gj_pair_kernel(Batch B, double* __restrict__ ws, int32_t* __restrict__ status, int with_rhs, int tr,
               long long wlim) {
  extern __shared__ __align__(16) char smem_raw[];
  PairPtrs P;
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int b = 2 * blockIdx.x + e;
    const Geo g = geo_of(B, b);
    const WsView w = ws_view(ws, g, B.ni, B.ld);
    P.Din[e] = w.inv;
    P.out[e] = w.inv;
    P.supn[e] = w.supn;
    P.subn[e] = w.subn;
    P.rhs[e] = with_rhs ? w.rmod : nullptr;
    P.status[e] = status + b;
  }
  gj_factor_pair<RPL, CPW, NW>(B.nz, B.ni, B.ld, P, tr != 0, smem_raw, wlim);
}

// out == nullptr: the inverses replace the blocks in the workspace (FP64
// path); otherwise they go to out (layer-major, ni x ld per layer) and the
// FP64 blocks stay. only != nullptr: atmospheres with only[b] == 0 are skipped.
template <int RPL, int CPW, int NW, int MB, bool DPF, typename R, bool PIPE = false>
__global__ void __launch_bounds__(NW * 32, MB)
gj_factor_kernel(Batch B, double* __restrict__ ws, R* out, const int32_t* __restrict__ only,
                 int32_t* __restrict__ status, int with_rhs, int tr, long long wlim, long long plim) {
  extern __shared__ __align__(16) char smem_raw[];
  const int b = blockIdx.x;
  if (only && only[b] == 0) return;
  Geo g = geo_of(B, b);
  WsView w = ws_view(ws, g, B.ni, B.ld);
  R* o = out ? out + g.z0 * B.ni * B.ld : reinterpret_cast<R*>(w.inv);
  gj_factor_atmosphere<RPL, CPW, NW, DPF, R, false, PIPE>(g.nz, B.ni, B.ld, w.inv, o, w.supn, w.subn,
                                                          with_rhs ? w.rmod : nullptr, tr != 0, status + b, smem_raw,
                                                          wlim, 0, nullptr, plim);
}

// FP32 factor of the mixed-precision step by the scalar Gauss-Jordan kernel
// (row-equilibrated, transposed orientation): FP32 inverses and row scales
// into the mixed region, the FP64 blocks stay in the workspace.
template <int RPL, int CPW, int NW, int MB, bool DPF, bool PIPE = false>
__global__ void __launch_bounds__(NW * 32, MB)
gj32_factor_kernel(Batch B, double* __restrict__ ws, void* __restrict__ mxr, int32_t* __restrict__ status,
                   long long wlim, long long plim) {
  extern __shared__ __align__(16) char smem_raw[];
  const int b = blockIdx.x;
  Geo g = geo_of(B, b);
  WsView w = ws_view(ws, g, B.ni, B.ld);
  MxView m = mx_view(mxr, g.z0, g.nz, B.ni);
  gj_factor_atmosphere<RPL, CPW, NW, DPF, float, true, PIPE>(g.nz, B.ni, B.ld, w.inv, m.X, w.supn, w.subn, nullptr,
                                                             true, status + b, smem_raw, wlim, round4(B.ni), m.rs,
                                                             plim);
}

// ---------------------------------------------------------------- blocked Gauss-Jordan factor (tensor cores)
// The same inverse as gj_factor_atmosphere (implicit partial pivoting,
// unnormalised pivot rows, result scattered to natural order), eliminated in
// panels of 8 columns, one warp per panel:
//  * Tile in registers in the mma accumulator layout: warp w holds columns
//    8w..8w+7 of B (B = A'^T when tr), lane (g = lane/4, t = lane%4) rows
//    8a+g (a < MR) and columns 8w+2t, 8w+2t+1: FP64 m8n8 accumulator tiles,
//    or (FP32) pairs of row groups forming m16n8 tiles.
//  * Panel q (columns 8q..8q+7): warp q runs its up to 8 pivot steps alone,
//    with warp-level communication only (argmax by redux.sync, pivot row and
//    column by shuffles), recording the multipliers m^(s)_i = S[i][k] / piv
//    of each step s (the mma A-operand layout) and the pivot rows p_s.
//  * Every other warp then applies the panel's 8 steps to its columns C at
//    once, as the right-looking blocked update (blocked LU's form)
//        U = L11^{-1} S[P, C]        (L11[s2][s] = m^(s)_{p_s2}, s < s2:
//                                     the pivot rows as they stood when they
//                                     pivoted; forward substitution)
//        S[:, C] -= M U              (M[i][s] = m^(s)_i: a rank-8 update,
//                                     mma.sync m8n8k4 FP64, or m16n8k8 TF32
//                                     with each operand split into a TF32
//                                     head and tail and three products
//                                     (head*head + head*tail + tail*head)
//                                     accumulated in FP32)
//    which equals the 8 single-pivot updates in exact arithmetic. The warp
//    that owns the next panel applies it to its own columns first and
//    starts that panel's pivot steps while the others update: one block
//    barrier per panel instead of one per pivot.
//  * EQ (FP32, tr): before the elimination every row of A'_j is scaled by a
//    power of two bringing its largest magnitude to [1, 2) (row
//    equilibration, exact); the stored inverse is X = (R A'_j)^{-1} with the
//    scales r, so A'_j^{-1} = X diag(r).
template <int NW, int MR, typename R>
struct BGJ {
  static constexpr int N = 8 * NW;   // padded columns (and rows of the FP64 tile)
  static constexpr int NR = 8 * MR;  // padded rows
  static constexpr int PBS = 12;     // column stride of a warp's pivot-row block
  static constexpr int MF = 2 * MR * 2 * 32;   // multiplier fragments of a panel (2 parities)
  static constexpr bool F32 = sizeof(R) == 4;
  __host__ __device__ static size_t al(size_t x) { return (x + 15) & ~(size_t)15; }
  static size_t smem_bytes(int n, int ld, int li, bool dpf) {
    return al((size_t)n * li * sizeof(R))                      // Ib: the inverse of the layer (natural order)
           + (dpf ? al((size_t)n * ld * sizeof(double)) : 0)   // Db: the next diagonal block, prefetched
           + al(MF * sizeof(R))                                // Mf: multipliers, A fragments
           + (F32 ? 2 * al(MF * sizeof(uint32_t)) : 0)         // TF32 head and tail of Mf
           + al(NW * 8 * PBS * sizeof(R))                      // Pb: per-warp pivot-row blocks
           + al(NR * sizeof(R))                                // rps: 1 / pivot of each row
           + al(2 * NR * sizeof(double))                       // rsb: the next layer's rhs and sub_d rows
           + al(2 * NR * sizeof(double))                       // vecs: right-hand side ping-pong
           + al(2 * N * sizeof(double))                        // rsc: row scales of this and the previous layer
           + al(N * sizeof(int))                               // pivs: pivot row of each step
           + al(NR * sizeof(int))                              // pslot: step at which each row pivoted (-1: not yet)
           + al(2 * 8 * sizeof(int))                           // ppan: pivot rows of a panel (2 parities; -1: none)
           + 16;                                               // mbarrier of the prefetch
  }
};

// D += A B for one m8n8k4 FP64 tile (A: 8x4 row, B: 4x8 col; per lane a0 =
// A[g][t], b0 = B[t][g], d = D[g][2t], D[g][2t+1]).
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// D += A B for one m16n8k8 TF32 tile (FP32 accumulation; per lane a = A[g][t],
// A[g+8][t], A[g][t+4], A[g+8][t+4]; b = B[t][g], B[t+4][g]; d = D[g][2t],
// D[g][2t+1], D[g+8][2t], D[g+8][2t+1]).
__device__ __forceinline__ void mma_tf32(float& d0, float& d1, float& d2, float& d3, uint32_t a0, uint32_t a1,
                                         uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d0), "+f"(d1), "+f"(d2), "+f"(d3)
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// TF32 head of x (round to nearest, ties away) and the TF32 head of the rest.
__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}

template <int NW, int MR, bool DPF, bool EQ, typename R>
__device__ __forceinline__ void bgj_factor_atmosphere(int nz, int n, int ld, int li, const double* Din, R* out,
                                                      double* rs_out, const double* __restrict__ supn,
                                                      const double* __restrict__ subn, double* rhs, bool tr,
                                                      int32_t* status, char* smem_raw, long long wlim) {
  using G = BGJ<NW, MR, R>;
  constexpr int N = G::N, NR = G::NR, PBS = G::PBS, MF = G::MF;
  constexpr bool F32 = G::F32;
  static_assert(!F32 || (MR % 2) == 0, "the FP32 tile pairs row groups into m16 tiles");
  static_assert(MR >= NW, "rows cover the columns");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const unsigned FULL = 0xffffffffu;
  const int dblk = n * ld, iblk = n * li;
  const int np = (n + 7) >> 3;   // panels holding columns of the block
  char* sp = smem_raw;
  auto take = [&](size_t bytes) {
    char* q = sp;
    sp += G::al(bytes);
    return q;
  };
  R* Ib = reinterpret_cast<R*>(take((size_t)iblk * sizeof(R)));
  double* Db = DPF ? reinterpret_cast<double*>(take((size_t)dblk * sizeof(double))) : nullptr;
  R* Mf = reinterpret_cast<R*>(take(MF * sizeof(R)));
  uint32_t* Mh = F32 ? reinterpret_cast<uint32_t*>(take(MF * sizeof(uint32_t))) : nullptr;
  uint32_t* Ml = F32 ? reinterpret_cast<uint32_t*>(take(MF * sizeof(uint32_t))) : nullptr;
  R* Pb = reinterpret_cast<R*>(take(NW * 8 * PBS * sizeof(R)));
  R* rps = reinterpret_cast<R*>(take(NR * sizeof(R)));
  double* rsb = reinterpret_cast<double*>(take(2 * NR * sizeof(double)));
  double* vecs = reinterpret_cast<double*>(take(2 * NR * sizeof(double)));
  double* rsc = reinterpret_cast<double*>(take(2 * N * sizeof(double)));
  int* pivs = reinterpret_cast<int*>(take(N * sizeof(int)));
  int* pslot = reinterpret_cast<int*>(take(NR * sizeof(int)));
  int* ppan = reinterpret_cast<int*>(take(2 * 8 * sizeof(int)));
  uint64_t* bar = reinterpret_cast<uint64_t*>(take(16));
  const uint32_t dbytes = (uint32_t)(dblk * sizeof(double));
  int st_local = 0;

  for (int e = threadIdx.x; e < iblk; e += blockDim.x) Ib[e] = R(0);   // padding columns stay 0
  if (rhs)
    for (int i = threadIdx.x; i < n; i += blockDim.x) vecs[i] = rhs[i];
  if (DPF && threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (DPF && threadIdx.x == 0) {
    mbar_expect_tx(bar, dbytes);
    bulk_g2s(Db, Din, dbytes, bar);
  }
  // multiplier m^(s)_r of the panel in buffer `buf` (A-fragment order)
  auto mval = [&](int buf, int r, int s) {
    return Mf[((buf * MR + (r >> 3)) * 2 + (s >> 2)) * 32 + (r & 7) * 4 + (s & 3)];
  };
  R acc[MR][2] = {};
  // value of row-slot a (warp-uniform or per-lane) of accumulator column e
  auto pick = [&](int a, int e) {
    R x = acc[0][e];
#pragma unroll
    for (int a2 = 1; a2 < MR; ++a2) x = (a == a2) ? acc[a2][e] : x;
    return x;
  };

  // Apply panel q's eliminations to this warp's columns (warp != q).
  auto apply_panel = [&](int q) {
    const int buf = q & 1;
    R* pb = Pb + warp * 8 * PBS;   // pb[c * PBS + s]: pivot row p_s, column c of this warp
#pragma unroll
    for (int a = 0; a < MR; ++a) {
      const int r = 8 * a + g;
      if (r < n) {
        const int sl = pslot[r];
        if (sl >= 0 && (sl >> 3) == q) {
          const int s = sl & 7;
          pb[(2 * t) * PBS + s] = acc[a][0];
          pb[(2 * t + 1) * PBS + s] = acc[a][1];
        }
      }
    }
    __syncwarp();
    if (lane < 8) {
      // forward substitution U = L11^{-1} S[P, c] for column c = lane; stored negated
      const int* pp = ppan + buf * 8;
      R u[8];
#pragma unroll
      for (int s = 0; s < 8; ++s) u[s] = pp[s] >= 0 ? pb[lane * PBS + s] : R(0);
#pragma unroll
      for (int s2 = 1; s2 < 8; ++s2) {
        const int r2 = pp[s2];
        if (r2 >= 0) {
#pragma unroll
          for (int s = 0; s < s2; ++s) u[s2] = fma(-mval(buf, r2, s), u[s], u[s2]);
        }
      }
#pragma unroll
      for (int s = 0; s < 8; ++s) pb[lane * PBS + s] = -u[s];
    }
    __syncwarp();
    const R b0 = pb[g * PBS + t], b1 = pb[g * PBS + 4 + t];
    if constexpr (!F32) {
      const R* mf = Mf + (size_t)buf * MR * 2 * 32;
#pragma unroll
      for (int a = 0; a < MR; ++a) {
        dmma_m8n8k4(acc[a][0], acc[a][1], mf[(a * 2 + 0) * 32 + lane], b0);
        dmma_m8n8k4(acc[a][0], acc[a][1], mf[(a * 2 + 1) * 32 + lane], b1);
      }
    } else {
      uint32_t bh0, bl0, bh1, bl1;
      tf32_split(b0, bh0, bl0);
      tf32_split(b1, bh1, bl1);
      const uint32_t* mh = Mh + (size_t)buf * MR * 2 * 32;
      const uint32_t* ml = Ml + (size_t)buf * MR * 2 * 32;
#pragma unroll
      for (int T = 0; T < MR / 2; ++T) {
        const int a0 = 2 * T, a1 = 2 * T + 1;
        const uint32_t h0 = mh[(a0 * 2 + 0) * 32 + lane], h1 = mh[(a1 * 2 + 0) * 32 + lane];
        const uint32_t h2 = mh[(a0 * 2 + 1) * 32 + lane], h3 = mh[(a1 * 2 + 1) * 32 + lane];
        const uint32_t l0 = ml[(a0 * 2 + 0) * 32 + lane], l1 = ml[(a1 * 2 + 0) * 32 + lane];
        const uint32_t l2 = ml[(a0 * 2 + 1) * 32 + lane], l3 = ml[(a1 * 2 + 1) * 32 + lane];
        mma_tf32(acc[a0][0], acc[a0][1], acc[a1][0], acc[a1][1], l0, l1, l2, l3, bh0, bh1);   // tail * head
        mma_tf32(acc[a0][0], acc[a0][1], acc[a1][0], acc[a1][1], h0, h1, h2, h3, bl0, bl1);   // head * tail
        mma_tf32(acc[a0][0], acc[a0][1], acc[a1][0], acc[a1][1], h0, h1, h2, h3, bh0, bh1);   // head * head
      }
    }
  };

  // Pivot steps of panel q in warp q (columns 8q + 2t + e of this warp).
  auto factor_panel = [&](int q) {
    const int buf = q & 1, k0 = 8 * q;
    const int cnt = min(8, n - k0);
    R* mf = Mf + (size_t)buf * MR * 2 * 32;
    unsigned used = 0;   // row slots a of this lane already pivoted (or padding)
#pragma unroll
    for (int a = 0; a < MR; ++a)
      if (8 * a + g >= n || pslot[8 * a + g] >= 0) used |= 1u << a;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      if (s < cnt) {
        const int te = s >> 1, ee = s & 1;
        const bool own = t == te;
        // ---- argmax of column s over the unpivoted rows (pivot_key32)
        unsigned km = 0u;
#pragma unroll
        for (int a = 0; a < MR; ++a) {
          const int r = 8 * a + g;
          if (own && r < n && !((used >> a) & 1u)) km = max(km, pivot_key32(acc[a][ee], r));
        }
        const int p = pivot_row(__reduce_max_sync(FULL, km));
        const R piv = __shfl_sync(FULL, pick(p >> 3, ee), ((p & 7) << 2) | te);
        if (piv == R(0)) st_local |= VB_STATUS_ZERO_PIVOT;
        const int ap = p >> 3, gp = p & 7;
        // column s to every lane of the quad, and this lane's part of row p
        R m[MR];
#pragma unroll
        for (int a = 0; a < MR; ++a) m[a] = __shfl_sync(FULL, acc[a][ee], (g << 2) | te);
        const R pr0 = __shfl_sync(FULL, pick(ap, 0), (gp << 2) | t);
        const R pr1 = __shfl_sync(FULL, pick(ap, 1), (gp << 2) | t);
        const R rp = rcp_rn(piv);
#pragma unroll
        for (int a = 0; a < MR; ++a) m[a] = (8 * a + g != p) ? m[a] * rp : R(0);
#pragma unroll
        for (int a = 0; a < MR; ++a) {
          acc[a][0] = fma(-m[a], pr0, acc[a][0]);
          acc[a][1] = fma(-m[a], pr1, acc[a][1]);
        }
#pragma unroll
        for (int a = 0; a < MR; ++a) {
          if (own) acc[a][ee] = (8 * a + g == p) ? R(1) : -m[a];
          if (t == (s & 3)) {
            const int fi = (a * 2 + (s >> 2)) * 32 + lane;
            mf[fi] = m[a];
            if constexpr (F32) tf32_split(m[a], Mh[buf * MR * 2 * 32 + fi], Ml[buf * MR * 2 * 32 + fi]);
          }
        }
        if (g == gp) used |= 1u << ap;
        if (lane == 0) {
          pivs[k0 + s] = p;
          rps[p] = rp;
          pslot[p] = k0 + s;
          ppan[buf * 8 + s] = p;
        }
      } else {
        // no step s: its multiplier column is zero
#pragma unroll
        for (int a = 0; a < MR; ++a)
          if (t == (s & 3)) {
            const int fi = (a * 2 + (s >> 2)) * 32 + lane;
            mf[fi] = R(0);
            if constexpr (F32) {
              Mh[buf * MR * 2 * 32 + fi] = 0u;
              Ml[buf * MR * 2 * 32 + fi] = 0u;
            }
          }
        if (lane == 0) ppan[buf * 8 + s] = -1;
      }
    }
  };

  for (int j = 0; j < nz; ++j) {
    if (DPF) {
      const bool ok = mbar_wait(bar, (uint32_t)(j & 1), wlim);
      if (__syncthreads_or(!ok)) {
        // give up: wait (bounded) for the copy still in flight, report, return
        if (threadIdx.x == 0) {
          mbar_wait(bar, (uint32_t)(j & 1), WAIT_LIMIT);
          atomicOr(status, VB_STATUS_WATCHDOG);
        }
        return;
      }
    }
    double rn = 0.0, sn = 0.0;
    const bool ride = rhs && j + 1 < nz && (int)threadIdx.x < n;
    if (ride) {
      rn = rhs[(int64_t)(j + 1) * n + threadIdx.x];
      sn = subn[(int64_t)j * n + threadIdx.x];
    }
    // ---- D_j and the Hadamard Schur update from Inv_{j-1} (solver.py:47):
    //      tile element (i, m) = B[i][m], A'_j[m][i] when tr, else A'_j[i][m]
    //      (EQ: Inv_{j-1} = X_{j-1} diag(r_{j-1}), and row m of A'_j is scaled)
    {
      const double* D = DPF ? Db : Din + (int64_t)j * dblk;
      const double* rprev = rsc + ((j + 1) & 1) * N;
      double sc[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int mcol = 8 * warp + 2 * t + e;
        sc[e] = (j > 0 && mcol < n) ? (tr ? subn : supn)[(int64_t)(j - 1) * n + mcol] : 0.0;
      }
      const int si = tr ? 1 : ld, sm = tr ? ld : 1;     // element strides of D (tile rows / columns)
      const int ii = tr ? 1 : li, im = tr ? li : 1;     // and of Ib
      double v[MR][2];
      double cmax[2] = {0.0, 0.0};
#pragma unroll
      for (int a = 0; a < MR; ++a) {
        const int i = 8 * a + g;
        const double sr = (j > 0 && i < n) ? (tr ? supn : subn)[(int64_t)(j - 1) * n + i] : 0.0;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int mcol = 8 * warp + 2 * t + e;
          double x = 0.0;
          if (i < n && mcol < n) {
            x = D[i * si + mcol * sm];
            if (j > 0) {
              const double cb = tr ? sc[e] * sr : sr * sc[e];
              double inv = (double)Ib[i * ii + mcol * im];
              if (EQ) inv = inv * rprev[i];
              x = x - cb * inv;
            }
          }
          v[a][e] = x;
          if (EQ) cmax[e] = fmax(cmax[e], fabs(x));
        }
      }
      if (EQ) {
        // largest magnitude of each tile column (row m of A'_j) over the 8 lanes sharing t
#pragma unroll
        for (int e = 0; e < 2; ++e)
#pragma unroll
          for (int off = 4; off < 32; off <<= 1) cmax[e] = fmax(cmax[e], __shfl_xor_sync(FULL, cmax[e], off));
        double* rcur = rsc + (j & 1) * N;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const double s = pow2_scale(cmax[e]);
          const int mcol = 8 * warp + 2 * t + e;
          if (g == 0 && mcol < n) {
            rcur[mcol] = s;
            rs_out[(int64_t)j * n + mcol] = s;
          }
#pragma unroll
          for (int a = 0; a < MR; ++a) v[a][e] *= s;
        }
      }
#pragma unroll
      for (int a = 0; a < MR; ++a) {
        acc[a][0] = (R)v[a][0];
        acc[a][1] = (R)v[a][1];
      }
    }
    for (int i = threadIdx.x; i < NR; i += blockDim.x) pslot[i] = -1;
    __syncthreads();   // Db and Ib consumed, pslot cleared
    if (DPF && threadIdx.x == 0 && j + 1 < nz) {
      fence_proxy_async();
      mbar_expect_tx(bar, dbytes);
      bulk_g2s(Db, Din + (int64_t)(j + 1) * dblk, dbytes, bar);
    }
    // ================================================================ elimination by panels
#pragma unroll 1
    for (int q = 0; q < np; ++q) {
      if (warp == q) {
        if (q > 0) apply_panel(q - 1);
        factor_panel(q);
      } else if (q > 0 && warp < np && warp != q - 1) {
        apply_panel(q - 1);
      }
      __syncthreads();
    }
    if (warp < np && warp != np - 1) apply_panel(np - 1);
    if (ride) {
      rsb[threadIdx.x] = rn;
      rsb[NR + threadIdx.x] = sn;
    }
    // ---- scale rows by 1/piv, scatter B^{-1}[q(i)][p_m] = T[i][m] into Ib
    //      (A'^{-1}[p_m][q(i)] when tr)
#pragma unroll
    for (int a = 0; a < MR; ++a) {
      const int i = 8 * a + g;
      if (i < n) {
        const R s = rps[i];
        const int qi = pslot[i];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int mcol = 8 * warp + 2 * t + e;
          if (mcol < n) {
            const R v = acc[a][e] * s;
            if (!isfinite(v)) st_local |= VB_STATUS_NONFINITE;
            Ib[tr ? pivs[mcol] * li + qi : qi * li + pivs[mcol]] = v;
          }
        }
      }
    }
    __syncthreads();
    // ---- Inv_j to global memory (natural order, padding columns 0)
    {
      using V = typename Pair<R>::T;
      V* O = reinterpret_cast<V*>(out + (int64_t)j * iblk);
      const V* S2 = reinterpret_cast<const V*>(Ib);
      for (int e = threadIdx.x; e < iblk / 2; e += blockDim.x) O[e] = S2[e];
    }
    // ---- forward sweep of the right-hand side: rhs[j+1] -= sub_d[j] o (Inv_j rhs[j])
    if (rhs && j + 1 < nz) {
      const double* vc = vecs + (j & 1) * NR;
      double* vn = vecs + ((j + 1) & 1) * NR;
      const int sub = lane & 3;
      for (int i0 = warp * 8; i0 < n; i0 += NW * 8) {
        const int i = i0 + (lane >> 2);
        double s0 = 0.0, s1 = 0.0;
        if (i < n) {
          int m2 = sub;
          for (; m2 + 4 < n; m2 += 8) {
            s0 = fma((double)Ib[i * li + m2], vc[m2], s0);
            s1 = fma((double)Ib[i * li + m2 + 4], vc[m2 + 4], s1);
          }
          if (m2 < n) s0 = fma((double)Ib[i * li + m2], vc[m2], s0);
        }
        double s = s0 + s1;
        s += __shfl_xor_sync(FULL, s, 1);
        s += __shfl_xor_sync(FULL, s, 2);
        if (sub == 0 && i < n) {
          const double v = rsb[i] - rsb[NR + i] * s;
          rhs[(int64_t)(j + 1) * n + i] = v;
          vn[i] = v;
        }
      }
    }
  }
  if (st_local) atomicOr(status, st_local);
}

// FP64: out == nullptr: the inverses replace the blocks in the workspace,
// otherwise they go to out (layer-major, ni x ld per layer). only != nullptr:
// atmospheres with only[b] == 0 are skipped.
template <int NW, int MB, bool DPF>
__global__ void __launch_bounds__(NW * 32, MB)
bgj_factor_kernel(Batch B, double* __restrict__ ws, double* out, const int32_t* __restrict__ only,
                  int32_t* __restrict__ status, int with_rhs, int tr, long long wlim) {
  extern __shared__ __align__(16) char smem_raw[];
  const int b = blockIdx.x;
  if (only && only[b] == 0) return;
  Geo g = geo_of(B, b);
  WsView w = ws_view(ws, g, B.ni, B.ld);
  double* o = out ? out + g.z0 * B.ni * B.ld : w.inv;
  bgj_factor_atmosphere<NW, NW, DPF, false, double>(g.nz, B.ni, B.ld, B.ld, w.inv, o, nullptr, w.supn, w.subn,
                                                     with_rhs ? w.rmod : nullptr, tr != 0, status + b, smem_raw,
                                                     wlim);
}

// FP32 factor of the mixed-precision step (row-equilibrated, transposed
// orientation): FP32 inverses and row scales into the mixed region.
template <int NW, int MR, int MB, bool DPF>
__global__ void __launch_bounds__(NW * 32, MB)
bgj32_factor_kernel(Batch B, double* __restrict__ ws, void* __restrict__ mxr, int32_t* __restrict__ status,
                    long long wlim) {
  extern __shared__ __align__(16) char smem_raw[];
  const int b = blockIdx.x;
  Geo g = geo_of(B, b);
  WsView w = ws_view(ws, g, B.ni, B.ld);
  MxView m = mx_view(mxr, g.z0, g.nz, B.ni);
  bgj_factor_atmosphere<NW, MR, DPF, true, float>(g.nz, B.ni, B.ld, round4(B.ni), w.inv, m.X, m.rs, w.supn, w.subn,
                                                   nullptr, true, status + b, smem_raw, wlim);
}

// ---------------------------------------------------------------- sweeps
constexpr int SWEEP_THREADS = 256;
constexpr int SWEEP_MAX_STAGES = 3;

__host__ __device__ inline size_t sweep_smem_bytes(int ni, int stages) {
  return (size_t)stages * ni * round_even(ni) * sizeof(double) + 64 + 2 * VB_MAX_NI * sizeof(double);
}

// out = Inv v (or Inv^T v) for one n x n block held in shared memory.
// Inv v: four lanes per row (two interleaved partial sums each, then two
// shuffle levels), eight rows per warp per pass; the pass loop is
// warp-uniform so every lane reaches the shuffles.
__device__ inline void block_matvec_s(const double* __restrict__ Inv, int n, int ld, bool trans,
                                      const double* v, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (!trans) {
    const int sub = lane & 3;
    for (int i0 = warp * 8; i0 < n; i0 += nw * 8) {
      const int i = i0 + (lane >> 2);
      double s0 = 0.0, s1 = 0.0;
      if (i < n) {
        const double* row = Inv + i * ld;
        int m = sub;
        for (; m + 4 < n; m += 8) {
          s0 = fma(row[m], v[m], s0);
          s1 = fma(row[m + 4], v[m + 4], s1);
        }
        if (m < n) s0 = fma(row[m], v[m], s0);
      }
      double s = s0 + s1;
      s += __shfl_xor_sync(0xffffffffu, s, 1);
      s += __shfl_xor_sync(0xffffffffu, s, 2);
      if (sub == 0 && i < n) out[i] = s;
    }
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double s = 0.0;
      for (int m = 0; m < n; ++m) s = fma(Inv[m * ld + i], v[m], s);
      out[i] = s;
    }
  }
}

// One sweep of one atmosphere over its stored inverses: forward elimination
// (solver.py:73-88) or back substitution (solver.py:91-111), optionally fused
// with the Ros2 combination (jax_step.py:313-314). The inverse blocks stream
// through a ring of `stages` shared-memory buffers filled by bulk copies.
__global__ void __launch_bounds__(SWEEP_THREADS)
sweep_kernel(Batch B, double* __restrict__ ws, SweepArgs A, int stages, long long wlim) {
  extern __shared__ __align__(128) char smem_raw[];
  const int b = blockIdx.x;
  Geo g = geo_of(B, b);
  WsView w = ws_view(ws, g, B.ni, B.ld);
  const int n = B.ni, nz = g.nz, ld = B.ld;
  const int blk = n * ld;
  const uint32_t blk_bytes = (uint32_t)(blk * sizeof(double));
  double* ring = reinterpret_cast<double*>(smem_raw);
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + (size_t)stages * blk);
  double* v = reinterpret_cast<double*>(bars + 8);
  double* u = v + VB_MAX_NI;
  const bool tr = A.transposed != 0;
  // transposed system: sub/super exchange roles (steady_state_grad.py:218-219)
  const double* up = tr ? w.subn : w.supn;   // couples x[j+1] into row j
  const double* lo = tr ? w.supn : w.subn;   // couples x[j-1] into row j
  double* vecs = A.user ? A.user + g.z0 * n : w.rmod;
  const bool fwd = A.mode == SWEEP_FWD;
  const int count = fwd ? nz - 1 : nz;                 // blocks used, in order
  auto block_of = [&](int s2) { return fwd ? s2 : nz - 1 - s2; };
  if (threadIdx.x == 0) {
    for (int st = 0; st < stages; ++st) mbar_init(&bars[st], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int st = 0; st < stages && st < count; ++st) {
      mbar_expect_tx(&bars[st], blk_bytes);
      bulk_g2s(ring + (size_t)st * blk, w.inv + (int64_t)block_of(st) * blk, blk_bytes, &bars[st]);
    }
  }
  double* out = A.user ? A.user + g.z0 * n : w.k1;
  const double r = ros2_r();
  const int tid = threadIdx.x;
  const bool own = tid < n;   // thread i owns element i of every vector (ni <= 128 < SWEEP_THREADS)
  if (fwd && own) v[tid] = vecs[tid];
  // Operands of a layer that do not depend on the running vector, loaded one
  // layer ahead so their latency hides behind the block copy and the product
  // (none of them is written by this kernel before it is read).
  double p_vec = 0.0, p_cpl = 0.0, p_y = 0.0, p_k1 = 0.0;
  auto prefetch = [&](int s2) {
    if (!own || s2 >= count) return;
    const int j = block_of(s2);
    if (fwd) {
      p_vec = vecs[(int64_t)(j + 1) * n + tid];
      p_cpl = lo[(int64_t)j * n + tid];
    } else {
      p_vec = vecs[(int64_t)j * n + tid];
      p_cpl = j < nz - 1 ? up[(int64_t)j * n + tid] : 0.0;
      if (A.mode == SWEEP_BACK_FINAL) {
        p_y = A.y[g.z0 * n + (int64_t)j * n + tid];
        p_k1 = w.k1[(int64_t)j * n + tid];
      }
    }
  };
  prefetch(0);
  int issued = min(stages, count);
  for (int s2 = 0; s2 < count; ++s2) {
    const int st = s2 % stages;
    const uint32_t parity = (uint32_t)((s2 / stages) & 1);
    const int j = block_of(s2);
    const double c_vec = p_vec, c_cpl = p_cpl, c_y = p_y, c_k1 = p_k1;
    prefetch(s2 + 1);
    if (!fwd && own) {
      double x = c_vec;
      if (j < nz - 1) x = x - c_cpl * u[tid];
      v[tid] = x;
    }
    const bool ok = mbar_wait(&bars[st], parity, wlim);
    if (__syncthreads_or(!ok)) {
      // give up: wait (bounded) for the copies still in flight, report, return
      if (threadIdx.x == 0) {
        for (int s3 = s2; s3 < issued; ++s3)
          mbar_wait(&bars[s3 % stages], (uint32_t)((s3 / stages) & 1), WAIT_LIMIT);
        if (A.status) atomicOr(A.status + b, VB_STATUS_WATCHDOG);
      }
      return;
    }
    block_matvec_s(ring + (size_t)st * blk, n, ld, tr, v, u);
    __syncthreads();
    if (threadIdx.x == 0 && s2 + stages < count) {
      fence_proxy_async();
      mbar_expect_tx(&bars[st], blk_bytes);
      bulk_g2s(ring + (size_t)st * blk, w.inv + (int64_t)block_of(s2 + stages) * blk, blk_bytes, &bars[st]);
      ++issued;
    }
    if (own) {
      if (fwd) {
        // rhs'[j+1] = rhs[j+1] - sub_d[j] o (Inv_j rhs'[j])
        const double x = c_vec - c_cpl * u[tid];
        vecs[(int64_t)(j + 1) * n + tid] = x;
        v[tid] = x;
      } else {
        const double kj = u[tid];
        if (A.mode == SWEEP_BACK) {
          out[(int64_t)j * n + tid] = kj;
        } else {
          // sol = y + 3/(2r) k1 + 1/(2r) k2 ; delta = |sol - yk2| (jax_step.py:313-314)
          const int64_t e = g.z0 * n + (int64_t)j * n + tid;
          const double s = c_y + (3.0 / (2.0 * r)) * c_k1 + (1.0 / (2.0 * r)) * kj;
          const double yk2 = c_y + c_k1 / r;
          w.aux[(int64_t)j * n + tid] = kj;   // k2, kept for vb_ros2_stages
          A.sol[e] = s;
          A.delta[e] = fabs(s - yk2);
          if (!isfinite(s)) atomicOr(A.status + b, VB_STATUS_NONFINITE);
        }
      }
    }
    __syncthreads();
  }
}

// Copy a uniform batch of dense blocks [B][nz][ni][ni] and off-diagonal
// vectors [B][nz-1][ni] into the factor layout.
__global__ void pack_blocks_kernel(Batch B, const double* __restrict__ diag, const double* __restrict__ sup_d,
                                   const double* __restrict__ sub_d, double* __restrict__ ws) {
  const int b = blockIdx.y, j = blockIdx.x;
  Geo g = geo_of(B, b);
  WsView w = ws_view(ws, g, B.ni, B.ld);
  const int n = B.ni;
  const double* src = diag + ((int64_t)b * g.nz + j) * n * n;
  double* dst = w.inv + (int64_t)j * n * B.ld;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e / n, c = e - i * n;
    dst[(int64_t)i * B.ld + c] = src[e];
  }
  if (j < g.nz - 1) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      w.supn[(int64_t)j * n + i] = sup_d[((int64_t)b * (g.nz - 1) + j) * n + i];
      w.subn[(int64_t)j * n + i] = sub_d[((int64_t)b * (g.nz - 1) + j) * n + i];
    }
  }
}

// FP64 FMA throughput probe: 8 independent dependent-FMA chains per thread.
__global__ void fp64_probe_kernel(double* out, int iters) {
  double a[8];
  const double m = 1.0000000001, c = 1e-12;
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * 1e-3 + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fma(a[k], m, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == 1234.5678) out[0] = s;  // keeps the loop live; practically never true
}

// ---------------------------------------------------------------- launchers
// Poll limit of the first bounded wait of each bulk copy; a wait that gives up
// drains the copies still in flight with the full WAIT_LIMIT before the CTA
// returns, so a lowered limit never leaves a copy writing to a finished CTA.
static long long g_wait_limit = WAIT_LIMIT;
void set_wait_limit(long long polls) { g_wait_limit = polls < 0 ? WAIT_LIMIT : polls; }
long long wait_limit() { return g_wait_limit; }
// Poll limit of the pipelined factor's step signals (every wait of the
// pipeline; giving up ends the atmosphere's factor with VB_STATUS_WATCHDOG).
static long long g_pipe_wait_limit = WAIT_LIMIT;
void set_pipe_wait_limit(long long polls) { g_pipe_wait_limit = polls < 0 ? WAIT_LIMIT : polls; }

cudaError_t launch_fp64_probe(double* out, int blocks, int threads, int iters, cudaStream_t st) {
  fp64_probe_kernel<<<blocks, threads, 0, st>>>(out, iters);
  return cudaGetLastError();
}

// SM count of the current device (the factor's layout depends on how many
// atmospheres share an SM).
static int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
    return 148;
  return n;
}

// One factor CTA per SM (the wider tile) or two: the tuning's choice, else
// one when the batch has at most one atmosphere per SM.
static bool one_cta_per_sm(const Batch& B) {
  if (B.factor_ctas) return B.factor_ctas == 1;
  return B.count <= sm_count();
}

template <int RPL, int CPW, int NW, int MB, bool DPF, typename R, bool PIPE>
static cudaError_t launch_gj_t(const Batch& B, double* ws, int32_t* status, int with_rhs, int tr, cudaStream_t st,
                               R* out, const int32_t* only) {
  size_t sm = GJK<RPL, CPW, NW, R>::smem_bytes(B.ni, B.ld, DPF, 0, PIPE);
  cudaError_t e = cudaFuncSetAttribute(gj_factor_kernel<RPL, CPW, NW, MB, DPF, R, PIPE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  gj_factor_kernel<RPL, CPW, NW, MB, DPF, R, PIPE><<<B.count, NW * 32, sm, st>>>(B, ws, out, only, status, with_rhs,
                                                                                       tr, g_wait_limit,
                                                                                       g_pipe_wait_limit);
  return cudaGetLastError();
}

// Factor kernel of the process: 0 = blocked Gauss-Jordan with the trailing
// updates on the FP64 tensor cores, 1 = scalar Gauss-Jordan with one block
// barrier per pivot step, 2 = scalar Gauss-Jordan pipelined per column panel
// (no block barrier per step), 3 = scalar Gauss-Jordan with two atmospheres'
// chains interleaved per CTA (FP64 factor of uniform batches of 65-72
// species; the scalar kernel elsewhere). A network's tuning (factor_kernel
// 1..4 = variant 0..3) overrides it.
static int g_factor_variant = 1;
void set_factor_variant(int v) { g_factor_variant = v; }
static int factor_choice(const Batch& B) { return B.factor_kernel ? B.factor_kernel - 1 : g_factor_variant; }

template <int NW, int MB, bool DPF>
static cudaError_t launch_bgj_t(const Batch& B, double* ws, int32_t* status, int with_rhs, int tr, cudaStream_t st,
                                double* out, const int32_t* only) {
  size_t sm = BGJ<NW, NW, double>::smem_bytes(B.ni, B.ld, B.ld, DPF);
  cudaError_t e = cudaFuncSetAttribute(bgj_factor_kernel<NW, MB, DPF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sm);
  if (e != cudaSuccess) return e;
  bgj_factor_kernel<NW, MB, DPF><<<B.count, NW * 32, sm, st>>>(B, ws, out, only, status, with_rhs, tr, g_wait_limit);
  return cudaGetLastError();
}

// Blocked factor shapes: one warp per 8-column panel (NW = ceil(ni / 8)
// rounded up to the instantiated sizes), the next diagonal block prefetched
// into shared memory where two copies fit.
static cudaError_t launch_bgj(const Batch& B, double* ws, int32_t* status, int with_rhs, int tr, cudaStream_t st,
                              double* out, const int32_t* only) {
  if (B.ni <= 32) return launch_bgj_t<4, 4, true>(B, ws, status, with_rhs, tr, st, out, only);
  if (B.ni <= 64) return launch_bgj_t<8, 2, true>(B, ws, status, with_rhs, tr, st, out, only);
  if (B.ni <= 72) {
    if (one_cta_per_sm(B)) return launch_bgj_t<9, 1, true>(B, ws, status, with_rhs, tr, st, out, only);
    return launch_bgj_t<9, 2, true>(B, ws, status, with_rhs, tr, st, out, only);
  }
  if (B.ni <= 96) return launch_bgj_t<12, 1, true>(B, ws, status, with_rhs, tr, st, out, only);
  return launch_bgj_t<16, 1, false>(B, ws, status, with_rhs, tr, st, out, only);
}

template <int NW, int MR, int MB, bool DPF>
static cudaError_t launch_bgj32_t(const Batch& B, double* ws, void* mxr, int32_t* status, cudaStream_t st) {
  size_t sm = BGJ<NW, MR, float>::smem_bytes(B.ni, B.ld, round4(B.ni), DPF);
  cudaError_t e = cudaFuncSetAttribute(bgj32_factor_kernel<NW, MR, MB, DPF>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  bgj32_factor_kernel<NW, MR, MB, DPF><<<B.count, NW * 32, sm, st>>>(B, ws, mxr, status, g_wait_limit);
  return cudaGetLastError();
}

template <int RPL, int CPW, int NW, int MB, bool DPF, bool PIPE>
static cudaError_t launch_gj32_t(const Batch& B, double* ws, void* mxr, int32_t* status, cudaStream_t st) {
  size_t sm = GJK<RPL, CPW, NW, float>::smem_bytes(B.ni, B.ld, DPF, round4(B.ni), PIPE);
  cudaError_t e = cudaFuncSetAttribute(gj32_factor_kernel<RPL, CPW, NW, MB, DPF, PIPE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  gj32_factor_kernel<RPL, CPW, NW, MB, DPF, PIPE><<<B.count, NW * 32, sm, st>>>(B, ws, mxr, status, g_wait_limit,
                                                                                      g_pipe_wait_limit);
  return cudaGetLastError();
}

template <bool PIPE>
static cudaError_t launch_gj32(const Batch& B, double* ws, void* mxr, int32_t* status32, cudaStream_t st) {
  if (B.ni <= 32) return launch_gj32_t<1, 4, 8, 4, true, PIPE>(B, ws, mxr, status32, st);
  if (B.ni <= 64) return launch_gj32_t<2, 8, 8, 2, true, PIPE>(B, ws, mxr, status32, st);
  if (B.ni <= 72) {
    if (one_cta_per_sm(B)) return launch_gj32_t<3, 6, 12, 1, true, PIPE>(B, ws, mxr, status32, st);
    return launch_gj32_t<3, 6, 12, 2, true, PIPE>(B, ws, mxr, status32, st);
  }
  return launch_gj32_t<3, 6, 16, 1, true, PIPE>(B, ws, mxr, status32, st);
}

cudaError_t launch_factor32(const Batch& B, double* ws, void* mxr, int32_t* status32, cudaStream_t st) {
  const int v = factor_choice(B);
  if (v == 1 || v == 3) return launch_gj32<false>(B, ws, mxr, status32, st);
  if (v == 2) return launch_gj32<true>(B, ws, mxr, status32, st);
  if (B.ni <= 32) return launch_bgj32_t<4, 4, 4, true>(B, ws, mxr, status32, st);
  if (B.ni <= 64) return launch_bgj32_t<8, 8, 2, true>(B, ws, mxr, status32, st);
  if (B.ni <= 72) {
    if (one_cta_per_sm(B)) return launch_bgj32_t<9, 10, 1, true>(B, ws, mxr, status32, st);
    return launch_bgj32_t<9, 10, 2, true>(B, ws, mxr, status32, st);
  }
  if (B.ni <= 96) return launch_bgj32_t<12, 12, 1, true>(B, ws, mxr, status32, st);
  return launch_bgj32_t<16, 16, 1, false>(B, ws, mxr, status32, st);
}



// Tile shapes by block size: rows over 32 lanes x RPL, columns over NW warps
// x CPW (the next diagonal block is prefetched into shared memory in every
// shape whose two buffers fit). Up to 72 species: 12 warps of 6 columns, two
// CTAs per SM when the batch has more atmospheres than SMs (register cap 85),
// else one (no register cap). Measured on B200, ni=69, nz=120: 148
// atmospheres 4.11 ms per factor (16 warps x 5: 4.77; 8 x 9: 5.30; 32 x 3:
// 6.43), one atmosphere 4.84 ms per Ros2 step (16 x 5: 5.50; 8 x 9: 5.92),
// 296 atmospheres 6.15 ms (two CTAs of 8 x 9: 6.29; 10 x 7: 6.15; 14 x 5:
// 7.09; 16 x 5: 9.14).
template <typename R, bool PIPE>
static cudaError_t launch_gj_p(const Batch& B, double* ws, int32_t* status, int with_rhs, int tr, cudaStream_t st,
                               R* out, const int32_t* only) {
  if (B.ni <= 32) return launch_gj_t<1, 4, 8, 4, true, R, PIPE>(B, ws, status, with_rhs, tr, st, out, only);
  if (B.ni <= 64) return launch_gj_t<2, 8, 8, 2, true, R, PIPE>(B, ws, status, with_rhs, tr, st, out, only);
  if (B.ni <= 72) {
    if (one_cta_per_sm(B))
      return launch_gj_t<3, 6, 12, 1, true, R, PIPE>(B, ws, status, with_rhs, tr, st, out, only);
    return launch_gj_t<3, 6, 12, 2, true, R, PIPE>(B, ws, status, with_rhs, tr, st, out, only);
  }
  // up to 96 species: 16 warps of 6 columns (the uneven 256-atmosphere batch,
  // whose ni=89 atmospheres set its floor: 16.49 ms per step against 16.99
  // with 12 warps of 8)
  if (B.ni <= 96) return launch_gj_t<3, 6, 16, 1, true, R, PIPE>(B, ws, status, with_rhs, tr, st, out, only);
  return launch_gj_t<4, 8, 16, 1, false, R, PIPE>(B, ws, status, with_rhs, tr, st, out, only);
}
template <typename R>
static cudaError_t launch_gj(const Batch& B, double* ws, int32_t* status, int with_rhs, int tr, cudaStream_t st,
                             R* out, const int32_t* only, bool pipe = false) {
  if (pipe) return launch_gj_p<R, true>(B, ws, status, with_rhs, tr, st, out, only);
  return launch_gj_p<R, false>(B, ws, status, with_rhs, tr, st, out, only);
}

// Paired factor: the pairs of atmospheres (2b, 2b+1), then an odd last
// atmosphere by the single kernel.
static cudaError_t launch_gj_pair(const Batch& B, double* ws, int32_t* status, int with_rhs, int tr,
                                  cudaStream_t st) {
  const size_t sm = GJP<3, 6, 12>::smem_bytes(B.ni, B.ld);
  cudaError_t e = cudaFuncSetAttribute(gj_pair_kernel<3, 6, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int pairs = B.count / 2;
  if (pairs > 0) gj_pair_kernel<3, 6, 12><<<pairs, 12 * 32, sm, st>>>(B, ws, status, with_rhs, tr, g_wait_limit);
  e = cudaGetLastError();
  if (e != cudaSuccess || (B.count & 1) == 0) return e;
  Batch B1 = B;
  B1.count = 1;
  const int64_t off = (int64_t)(B.count - 1) * B.nz * ws_per_layer(B.ni, B.ld);
  return launch_gj_t<3, 6, 12, 1, true, double, false>(B1, ws + off, status + (B.count - 1), with_rhs, tr, st,
                                                       nullptr, nullptr);
}
static bool pair_applies(const Batch& B) { return !B.zoff && B.ni > 64 && B.ni <= 72 && B.count >= 2; }

cudaError_t launch_factor_only(const Batch& B, double* ws, const int32_t* only, int32_t* status, cudaStream_t st) {
  const int v = factor_choice(B);
  if (v == 0) return launch_bgj(B, ws, status, 0, 1, st, nullptr, only);
  return launch_gj<double>(B, ws, status, 0, 1, st, nullptr, only, v == 2);
}

cudaError_t launch_factor(const Batch& B, double* ws, int32_t* status, int with_rhs, cudaStream_t st,
                          bool for_transposed_solves) {
  const int tr = for_transposed_solves ? 0 : 1;
  const int v = factor_choice(B);
  if (v == 0) return launch_bgj(B, ws, status, with_rhs, tr, st, nullptr, nullptr);
  if (v == 3 && pair_applies(B)) return launch_gj_pair(B, ws, status, with_rhs, tr, st);
  return launch_gj<double>(B, ws, status, with_rhs, tr, st, nullptr, nullptr, v == 2);
}

// Factors into a separate inverse region (the workspace keeps the FP64
// blocks): R = float for the mixed-precision solve, R = double for its FP64
// fallback (only the atmospheres with only[b] != 0).
template <typename R>
cudaError_t launch_factor_into(const Batch& B, double* ws, R* out, const int32_t* only, int32_t* status,
                               cudaStream_t st) {
  return launch_gj<R>(B, ws, status, 0, 1, st, out, only);
}
template cudaError_t launch_factor_into<float>(const Batch&, double*, float*, const int32_t*, int32_t*, cudaStream_t);
template <>
cudaError_t launch_factor_into<double>(const Batch& B, double* ws, double* out, const int32_t* only, int32_t* status,
                                       cudaStream_t st) {
  const int v = factor_choice(B);
  if (v == 0) return launch_bgj(B, ws, status, 0, 1, st, out, only);
  return launch_gj<double>(B, ws, status, 0, 1, st, out, only, v == 2);
}

cudaError_t launch_sweep(const Batch& B, double* ws, const SweepArgs& A, cudaStream_t st) {
  int stages = B.sweep_stages ? B.sweep_stages : SWEEP_MAX_STAGES;
  while (stages > 1 && sweep_smem_bytes(B.ni, stages) > 220 * 1024) --stages;
  // more atmospheres than SMs: a shallower ring lets two CTAs share an SM (one wave)
  if (!B.sweep_stages && B.count > sm_count())
    while (stages > 2 && 2 * sweep_smem_bytes(B.ni, stages) > 224 * 1024) --stages;
  size_t sm = sweep_smem_bytes(B.ni, stages);
  cudaError_t e = cudaFuncSetAttribute(sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  sweep_kernel<<<B.count, SWEEP_THREADS, sm, st>>>(B, ws, A, stages, g_wait_limit);
  return cudaGetLastError();
}

cudaError_t launch_pack_blocks(const Batch& B, const double* diag, const double* sup_d,
                               const double* sub_d, double* ws, cudaStream_t st) {
  dim3 grid(B.nz, B.count);
  pack_blocks_kernel<<<grid, 256, 0, st>>>(B, diag, sup_d, sub_d, ws);
  return cudaGetLastError();
}

}  // namespace vb
