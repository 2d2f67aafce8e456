// Block-tridiagonal Thomas for dense diagonal blocks and diagonal off-diagonal
// blocks (reference solver.py:33-126), one persistent CTA per atmosphere.
//
// factor: for each layer j (serial in z)
//     A'_j  = D_j - (sub_d[j-1] sup_d[j-1]^T) o A'_{j-1}^{-1}     (solver.py:47)
//     Inv_j = A'_j^{-1}                                            (solver.py:46,48)
// The inverse is formed by Gauss-Jordan elimination with partial pivoting on
// a register-resident tile (each warp owns RPW rows, each lane NP/32 columns),
// with implicit row pivoting (no row exchanges; the permutation is undone when
// the tile is stored). The forward sweep of the first right-hand side rides
// along (solver.py:73-88). The stored inverses turn every later solve into
// matrix-vector products (solver.py:91-111).
#include <cuda_runtime.h>

#include "vb_common.cuh"
#include "vb_launch.cuh"

namespace vb {

template <int NP, int NW, int PW>
struct LUK {
  static constexpr int RPW = NP / NW;     // rows per warp
  static constexpr int CPL = NP / 32;     // columns per lane
  static constexpr int PRL = NP / 32;     // panel rows per lane of the panel warp
  static constexpr int SLD = NP + 1;      // smem row stride of S (doubles)
  static constexpr int PLD = PW + 1;      // smem row stride of a panel buffer
  static constexpr int PBUF = (NP * PLD > RPW * NP) ? NP * PLD : RPW * NP;
  static size_t smem_bytes() {
    size_t d = (size_t)NP * SLD          // S: previous inverse, LU factors, new inverse
               + 2 * (size_t)PBUF        // panel buffers / triangular-solve row buffers
               + (size_t)NP * PLD        // M: update multipliers of the current panel
               + (size_t)PW * NP         // V: pivot rows of the current panel
               + 2 * (size_t)NP          // vec, rdiag
               + PW + PW * PW;           // pivot row broadcast, L_KK^{-1}
    return d * sizeof(double) + sizeof(int) * 2 * NP;
  }
};

// Pivot key of a candidate: |v| as an order-preserving 64-bit pattern (NaN -> 0).
__device__ __forceinline__ unsigned long long pivot_key(double v) {
  double a = fabs(v);
  return (a >= 0.0) ? (unsigned long long)__double_as_longlong(a) : 0ull;
}

// Factor all layers of one atmosphere. On entry inv[j] holds D_j (row stride
// ld); on exit inv[j] holds A'_j^{-1}. With rhs != nullptr the first sweep of
// the right-hand side rhs[nz][ni] is done in place (solver.py:73-88).
//
// Each diagonal block is inverted as the reference does (solver.py:46-48):
// LU with partial pivoting (lu_factor), then the inverse by forward and back
// substitution on the identity (lu_solve(LU, I)).
//  * LU: blocked right-looking elimination with implicit row pivoting on a
//    register-resident tile (warp w owns rows w*RPW.., lane l columns l+32c).
//    Warp 0 factors each PW-column panel (argmax over unpivoted rows by three
//    redux.sync reductions, pivot row broadcast through shared memory);
//    every warp then forms U[K, C] = L_KK^{-1} A[P, C] for its columns and
//    applies the rank-PW update A[R, C] -= L[R, K] U[K, C] to unpivoted rows.
//  * The factors are stored in pivot order in shared memory; the tile is
//    re-used for Y = L^{-1} P and X = U^{-1} Y, one warp's RPW rows per
//    panel (solved thread-locally, then broadcast and applied by the other
//    warps), so X = A'^{-1} ends up in natural row order.
template <int NP, int NW, int PW>
__device__ void factor_atmosphere(int nz, int n, int ld, double* __restrict__ inv,
                                  const double* __restrict__ supn, const double* __restrict__ subn,
                                  double* __restrict__ rhs, int32_t* status, char* smem_raw) {
  using G = LUK<NP, NW, PW>;
  constexpr int RPW = G::RPW, CPL = G::CPL, PRL = G::PRL, SLD = G::SLD, PLD = G::PLD;
  double* S = reinterpret_cast<double*>(smem_raw);          // [NP][SLD]
  double* Pn0 = S + NP * SLD;                               // [PBUF]
  double* Pn1 = Pn0 + G::PBUF;                              // [PBUF]
  double* Mb = Pn1 + G::PBUF;                               // [NP][PLD]
  double* V = Mb + NP * PLD;                                // [PW][NP]
  double* vec = V + PW * NP;                                // [NP]
  double* rdiag = vec + NP;                                 // [NP]
  double* prow_s = rdiag + NP;                              // [PW]
  double* Linv = prow_s + PW;                               // [PW][PW]
  int* pivs = reinterpret_cast<int*>(Linv + PW * PW);       // [NP] pivot row of step k
  int* qinv = pivs + NP;                                    // [NP] step of row i (-1: not yet)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned FULL = 0xffffffffu;
  int st_local = 0;

  if (rhs) {
    for (int i = threadIdx.x; i < NP; i += blockDim.x) vec[i] = i < n ? rhs[i] : 0.0;
  }
  const int npan = (n + PW - 1) / PW;

  double a[RPW][CPL];
  for (int j = 0; j < nz; ++j) {
    const double* D = inv + (int64_t)j * n * ld;
    for (int i = threadIdx.x; i < NP; i += blockDim.x) qinv[i] = -1;
    // ---- load D_j and apply the Hadamard Schur update from Inv_{j-1} (solver.py:47)
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
      int i = warp * RPW + r;
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        int col = lane + 32 * c;
        double v = 0.0;
        if (i < n && col < n) {
          v = D[(int64_t)i * ld + col];
          if (j > 0) {
            double cb = subn[(int64_t)(j - 1) * n + i] * supn[(int64_t)(j - 1) * n + col];
            v = v - cb * S[i * SLD + col];
          }
        }
        a[r][c] = v;
      }
    }
    unsigned usedw = 0;     // warp 0: rows lane + 32*r already pivoted
    // ================================================================ LU
    for (int pb = 0; pb < npan; ++pb) {
      const int k0 = pb * PW;
      const int kw = min(PW, n - k0);
      double* Pn = (pb & 1) ? Pn1 : Pn0;
      // (a) owners of the panel columns stage them
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        int col = lane + 32 * c;
        if (col >= k0 && col < k0 + PW) {
#pragma unroll
          for (int r = 0; r < RPW; ++r) Pn[(warp * RPW + r) * PLD + (col - k0)] = a[r][c];
        }
      }
      __syncthreads();
      // (b) warp 0: unblocked LU of the panel (in shared memory) over the
      //     unpivoted rows, then L_KK^{-1} of its unit lower triangle
      if (warp == 0) {
#pragma unroll
        for (int t = 0; t < PW; ++t) {
          if (t < kw) {
            unsigned long long bk = 0ull;
            unsigned brow = 0xffffffffu;
#pragma unroll
            for (int r = 0; r < PRL; ++r) {
              const int i = lane + 32 * r;
              if (i < n && !((usedw >> r) & 1u)) {
                unsigned long long kk = pivot_key(Pn[i * PLD + t]);
                if (brow == 0xffffffffu || kk > bk) { bk = kk; brow = (unsigned)i; }
              }
            }
            const unsigned hi = (unsigned)(bk >> 32), lo = (unsigned)bk;
            const unsigned m1 = __reduce_max_sync(FULL, hi);
            const unsigned m2 = __reduce_max_sync(FULL, hi == m1 ? lo : 0u);
            const int p = (int)__reduce_min_sync(FULL, (hi == m1 && lo == m2) ? brow : 0xffffffffu);
            if ((p & 31) == lane) usedw |= 1u << (p >> 5);
            const double* prow = Pn + p * PLD;
            const double piv = prow[t];
            if (piv == 0.0) st_local |= VB_STATUS_ZERO_PIVOT;
            const double rcp = 1.0 / piv;
            double pr[PW];
#pragma unroll
            for (int u = t + 1; u < PW; ++u) pr[u] = prow[u];
#pragma unroll
            for (int r = 0; r < PRL; ++r) {
              const int i = lane + 32 * r;
              if (i < n && !((usedw >> r) & 1u)) {
                double* row = Pn + i * PLD;
                const double l = row[t] * rcp;
                row[t] = l;
#pragma unroll
                for (int u = t + 1; u < PW; ++u) row[u] = fma(-l, pr[u], row[u]);
              }
            }
            if (lane == 0) { pivs[k0 + t] = p; qinv[p] = k0 + t; }
            __syncwarp();
          }
        }
        // L_KK^{-1} (unit lower): lane s builds column s from the pivot rows' multipliers
        if (lane < PW) {
          const int sc = lane;
          double li[PW];
#pragma unroll
          for (int t = 0; t < PW; ++t) {
            double x = (t == sc) ? 1.0 : 0.0;
            if (t > sc && t < kw) {
              const double* lrow = Pn + pivs[k0 + t] * PLD;
#pragma unroll
              for (int m = 0; m < t; ++m)
                if (m >= sc) x = fma(-lrow[m], li[m], x);
            }
            li[t] = x;
          }
#pragma unroll
          for (int t = 0; t < PW; ++t) Linv[t * PW + sc] = li[t];
        }
      }
      __syncthreads();
      // (b') every warp: update multipliers of its own rows. Unpivoted rows
      //     M = -L[i,K] L_KK^{-1}; pivot row p_t: M = L_KK^{-1}[t,:] - e_t (so
      //     W + M V = U[t,:]); rows pivoted earlier: 0.
      for (int e = lane; e < RPW * PW; e += 32) {
        const int r = e / PW, u = e - r * PW;
        const int i = warp * RPW + r;
        const int q = i < n ? qinv[i] : -2;
        double x = 0.0;
        if (i < n && q < 0) {
          const double* row = Pn + i * PLD;
#pragma unroll
          for (int s2 = 0; s2 < PW; ++s2)
            if (s2 >= u && s2 < kw) x = fma(-row[s2], Linv[s2 * PW + u], x);
        } else if (q >= k0 && q < k0 + kw) {
          const int t = q - k0;
          x = (u <= t) ? Linv[t * PW + u] - (u == t ? 1.0 : 0.0) : 0.0;
        }
        Mb[i * PLD + u] = x;
      }
      // (c) owners of the new pivot rows stage them: V[t] = A[p_t, :]
#pragma unroll
      for (int r = 0; r < RPW; ++r) {
        int i = warp * RPW + r;
        int q = qinv[i];
        if (q >= k0 && q < k0 + kw) {
#pragma unroll
          for (int c = 0; c < CPL; ++c) V[(q - k0) * NP + lane + 32 * c] = a[r][c];
        }
      }
      __syncthreads();
      // (d) rank-kw update A[i, C] += M[i, K] V[K, C] (C = columns right of the
      //     panel): unpivoted rows get the Schur update, pivot rows become
      //     U[K, C] = L_KK^{-1} V; rows pivoted in earlier panels are final.
#pragma unroll
      for (int r = 0; r < RPW; ++r) {
        const int i = warp * RPW + r;
        const int q = qinv[i];
        if (q >= 0 && q < k0) continue;
        double mi[PW];
#pragma unroll
        for (int t = 0; t < PW; ++t) mi[t] = Mb[i * PLD + t];
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          const int col = lane + 32 * c;
          if (col >= k0 && col < k0 + PW) {
            a[r][c] = Pn[i * PLD + (col - k0)];
          } else if (col >= k0 + PW) {
            double acc = a[r][c];
#pragma unroll
            for (int t = 0; t < PW; ++t)
              if (t < kw) acc = fma(mi[t], V[t * NP + col], acc);
            a[r][c] = acc;
          }
        }
      }
    }
    // ---- factors to shared memory in pivot order (LAPACK layout), 1/U_kk
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
      int i = warp * RPW + r;
      if (i < n) {
        int qi = qinv[i];
#pragma unroll
        for (int c = 0; c < CPL; ++c) S[qi * SLD + lane + 32 * c] = a[r][c];
      }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) rdiag[k] = 1.0 / S[k * SLD + k];
    // ================================================================ Y = L^{-1} P
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
      const int k = warp * RPW + r;
      const int pk = k < n ? pivs[k] : -1;
#pragma unroll
      for (int c = 0; c < CPL; ++c) a[r][c] = (lane + 32 * c == pk) ? 1.0 : 0.0;
    }
    for (int w = 0; w < NW; ++w) {
      const int k0 = w * RPW;
      if (k0 >= n) break;
      double* Yb = (w & 1) ? Pn1 : Pn0;
      if (warp == w) {
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
          const int k = k0 + r;
#pragma unroll
          for (int s2 = 0; s2 < r; ++s2) {
            const double l = k < n ? S[k * SLD + k0 + s2] : 0.0;
#pragma unroll
            for (int c = 0; c < CPL; ++c) a[r][c] = fma(-l, a[s2][c], a[r][c]);
          }
#pragma unroll
          for (int c = 0; c < CPL; ++c) Yb[r * NP + lane + 32 * c] = a[r][c];
        }
      }
      __syncthreads();
      if (warp > w) {
        const int kw = min(RPW, n - k0);
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
          const int k = warp * RPW + r;
          if (k < n) {
#pragma unroll
            for (int s2 = 0; s2 < RPW; ++s2) {
              if (s2 < kw) {
                const double l = S[k * SLD + k0 + s2];
#pragma unroll
                for (int c = 0; c < CPL; ++c) a[r][c] = fma(-l, Yb[s2 * NP + lane + 32 * c], a[r][c]);
              }
            }
          }
        }
      }
    }
    // ================================================================ X = U^{-1} Y
    __syncthreads();   // readers of the forward phase's last buffer are done
    for (int w = NW - 1; w >= 0; --w) {
      const int k0 = w * RPW;
      if (k0 >= n) continue;
      const int kw = min(RPW, n - k0);
      double* Yb = (w & 1) ? Pn1 : Pn0;   // last read two panels ago, before the previous barrier
      if (warp == w) {
#pragma unroll
        for (int r = RPW - 1; r >= 0; --r) {
          const int k = k0 + r;
          if (r < kw) {
#pragma unroll
            for (int s2 = r + 1; s2 < RPW; ++s2) {
              if (s2 < kw) {
                const double uu = S[k * SLD + k0 + s2];
#pragma unroll
                for (int c = 0; c < CPL; ++c) a[r][c] = fma(-uu, a[s2][c], a[r][c]);
              }
            }
            const double rd = rdiag[k];
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
              a[r][c] = a[r][c] * rd;
              Yb[r * NP + lane + 32 * c] = a[r][c];
            }
          }
        }
      }
      __syncthreads();
      if (warp < w) {
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
          const int k = warp * RPW + r;
          if (k < n) {
#pragma unroll
            for (int s2 = 0; s2 < RPW; ++s2) {
              if (s2 < kw) {
                const double uu = S[k * SLD + k0 + s2];
#pragma unroll
                for (int c = 0; c < CPL; ++c) a[r][c] = fma(-uu, Yb[s2 * NP + lane + 32 * c], a[r][c]);
              }
            }
          }
        }
      }
    }
    // ---- the inverse (natural order) to shared and global memory
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
      int i = warp * RPW + r;
      if (i < n) {
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          int col = lane + 32 * c;
          if (col < n) {
            if (!isfinite(a[r][c])) st_local |= VB_STATUS_NONFINITE;
            S[i * SLD + col] = a[r][c];
          }
        }
      }
    }
    __syncthreads();
    double* O = inv + (int64_t)j * n * ld;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      int i = e / n, col = e - i * n;
      O[(int64_t)i * ld + col] = S[i * SLD + col];
    }
    // ---- forward sweep of the right-hand side: rhs[j+1] -= sub_d[j] o (Inv_j rhs[j])
    if (rhs && j + 1 < nz) {
      double* u = Pn0;
      for (int i = warp; i < n; i += NW) {
        double s = 0.0;
        for (int m = lane; m < n; m += 32) s += S[i * SLD + m] * vec[m];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(FULL, s, off);
        if (lane == 0) u[i] = s;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double v = rhs[(int64_t)(j + 1) * n + i] - subn[(int64_t)j * n + i] * u[i];
        rhs[(int64_t)(j + 1) * n + i] = v;
        vec[i] = v;
      }
    }
    __syncthreads();
  }
  if (st_local) atomicOr(status, st_local);
}

template <int NP, int NW, int PW>
__global__ void __launch_bounds__(NW * 32, 1)
factor_kernel(Batch B, double* __restrict__ ws, int32_t* __restrict__ status, int with_rhs) {
  extern __shared__ __align__(16) char smem_raw[];
  const int b = blockIdx.x;
  Geo g = geo_of(B, b);
  WsView w = ws_view(ws, g, B.ni, B.ld);
  factor_atmosphere<NP, NW, PW>(g.nz, B.ni, B.ld, w.inv, w.supn, w.subn, with_rhs ? w.rmod : nullptr,
                                status + b, smem_raw);
}

// ---------------------------------------------------------------- sweeps
constexpr int SWEEP_THREADS = 256;
constexpr int SWEEP_MAX_STAGES = 3;

__host__ __device__ inline size_t sweep_smem_bytes(int ni, int stages) {
  return (size_t)stages * ni * round_even(ni) * sizeof(double) + 64 + 2 * VB_MAX_NI * sizeof(double);
}

// out = Inv v (or Inv^T v) for one n x n block held in shared memory.
__device__ inline void block_matvec_s(const double* __restrict__ Inv, int n, int ld, bool trans,
                                      const double* v, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (!trans) {
    for (int i = warp; i < n; i += nw) {
      double s = 0.0;
      for (int m = lane; m < n; m += 32) s = fma(Inv[i * ld + m], v[m], s);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      if (lane == 0) out[i] = s;
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
sweep_kernel(Batch B, double* __restrict__ ws, SweepArgs A, int stages) {
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
  if (fwd) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) v[i] = vecs[i];
  }
  int issued = min(stages, count);
  for (int s2 = 0; s2 < count; ++s2) {
    const int st = s2 % stages;
    const uint32_t parity = (uint32_t)((s2 / stages) & 1);
    const int j = block_of(s2);
    if (!fwd) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double x = vecs[(int64_t)j * n + i];
        if (j < nz - 1) x = x - up[(int64_t)j * n + i] * u[i];
        v[i] = x;
      }
    }
    const bool ok = mbar_wait(&bars[st], parity, WAIT_LIMIT);
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
    if (fwd) {
      // rhs'[j+1] = rhs[j+1] - sub_d[j] o (Inv_j rhs'[j])
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double x = vecs[(int64_t)(j + 1) * n + i] - lo[(int64_t)j * n + i] * u[i];
        vecs[(int64_t)(j + 1) * n + i] = x;
        v[i] = x;
      }
    } else {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double kj = u[i];
        if (A.mode == SWEEP_BACK) {
          out[(int64_t)j * n + i] = kj;
        } else {
          // sol = y + 3/(2r) k1 + 1/(2r) k2 ; delta = |sol - yk2| (jax_step.py:313-314)
          int64_t e = g.z0 * n + (int64_t)j * n + i;
          double yv = A.y[e];
          double k1v = w.k1[(int64_t)j * n + i];
          double s = yv + (3.0 / (2.0 * r)) * k1v + (1.0 / (2.0 * r)) * kj;
          double yk2 = yv + k1v / r;
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
cudaError_t launch_fp64_probe(double* out, int blocks, int threads, int iters, cudaStream_t st) {
  fp64_probe_kernel<<<blocks, threads, 0, st>>>(out, iters);
  return cudaGetLastError();
}

template <int NP, int NW, int PW>
static cudaError_t launch_factor_t(const Batch& B, double* ws, int32_t* status, int with_rhs,
                                   cudaStream_t st) {
  size_t sm = LUK<NP, NW, PW>::smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(factor_kernel<NP, NW, PW>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  factor_kernel<NP, NW, PW><<<B.count, NW * 32, sm, st>>>(B, ws, status, with_rhs);
  return cudaGetLastError();
}

cudaError_t launch_factor(const Batch& B, double* ws, int32_t* status, int with_rhs, cudaStream_t st) {
  if (B.ni <= 32) return launch_factor_t<32, 8, 8>(B, ws, status, with_rhs, st);
  if (B.ni <= 64) return launch_factor_t<64, 16, 8>(B, ws, status, with_rhs, st);
  if (B.ni <= 96) return launch_factor_t<96, 16, 8>(B, ws, status, with_rhs, st);
  return launch_factor_t<128, 16, 8>(B, ws, status, with_rhs, st);
}

cudaError_t launch_sweep(const Batch& B, double* ws, const SweepArgs& A, cudaStream_t st) {
  int stages = SWEEP_MAX_STAGES;
  while (stages > 1 && sweep_smem_bytes(B.ni, stages) > 220 * 1024) --stages;
  size_t sm = sweep_smem_bytes(B.ni, stages);
  cudaError_t e = cudaFuncSetAttribute(sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  sweep_kernel<<<B.count, SWEEP_THREADS, sm, st>>>(B, ws, A, stages);
  return cudaGetLastError();
}

cudaError_t launch_pack_blocks(const Batch& B, const double* diag, const double* sup_d,
                               const double* sub_d, double* ws, cudaStream_t st) {
  dim3 grid(B.nz, B.count);
  pack_blocks_kernel<<<grid, 256, 0, st>>>(B, diag, sup_d, sub_d, ws);
  return cudaGetLastError();
}

}  // namespace vb
