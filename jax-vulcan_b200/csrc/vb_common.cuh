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
  // RHS gather tables: for species i, the (r*T+s) slots whose reactant (loss)
  // or product (prod) index is i, in increasing flat order (segment_sum order).
  const int32_t* loss_ptr;       // [ni+1]
  const int32_t* loss_ent;
  const int32_t* prod_ptr;       // [ni+1]
  const int32_t* prod_ent;
  // Jacobian gather table: for destination d = row*ni+col, the flat contribution
  // indices e = (r*2T + o)*T + s in increasing order (chem.py:193-207 scatter order).
  const int32_t* jac_ptr;        // [ni*ni+1]
  const int32_t* jac_ent;
};

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
};

struct Geo {
  int nz;
  int64_t z0;        // first layer of this atmosphere in the packed layer axis
  int64_t atm;       // blob offset (doubles)
  int64_t ws;        // workspace offset (doubles)
};

// Workspace doubles per layer: inverse block + rmod + k1 + sup_neg + sub_neg + spare.
__host__ __device__ inline int64_t ws_per_layer(int ni, int ld) {
  return (int64_t)ni * ld + 5 * (int64_t)ni;
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

// Ros2 constants (reference jax_step.py:257-258).
__device__ __forceinline__ double ros2_r() { return 1.0 + 1.0 / sqrt(2.0); }

}  // namespace vb
