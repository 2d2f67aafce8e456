// One attempt of the adaptive loop body after a Ros2 step (reference
// outer_loop.py:715-1100, the parts that decide the step): fixed species
// (:733-739), clip (_make_clip_fn :196-224), atom loss (_compute_atom_loss
// :171-178), error norm (_make_aggregate_delta_fn :227-250), accept /
// force-accept (:745-756), reject counters (:758-764), time (:766-768),
// hydrostatic rebalance (:844-853), next y / ymix / atom loss (:899-917),
// adaptive rtol (:990-1020) and the next dt (_step_size :181-193,
// :1022-1031). An atmosphere whose convergence record is done is skipped.
//
// loop_conv_kernel, after the body: ring buffer of (y, t), the lookback and
// the relative change longdy / longdydt, the stall counter, the
// photo-frequency switch and the loop condition, per atmosphere.
//
// One CTA per atmosphere, one warp per layer (lanes over species, ni <= 128).
// Phase A clips and reduces (error norm, sign flags, clipped mass, per-layer
// ysums kept in shared memory, per-atom sums); thread 0 decides; phase B
// rewrites y / y_prev / ymix from the same per-element arithmetic. Every
// decision is CTA-uniform and stays on the device, so a loop of step + body
// needs no host round trip. Compiled with --fmad=false (element-wise
// rounding as the reference's NumPy/XLA expressions).
#include <cuda_runtime.h>

#include "vb_common.cuh"
#include "vb_launch.cuh"

namespace vb {

constexpr int BODY_THREADS = 256;
constexpr int BODY_WARPS = BODY_THREADS / 32;

// jnp.maximum / jnp.minimum: NaN propagates.
__device__ __forceinline__ double jmax(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }
__device__ __forceinline__ double jmin(double a, double b) { return (a != a || b != b) ? a + b : fmin(a, b); }

__device__ __forceinline__ double step_size(double dt, double delta, double rtol, const VbLoopParams& p) {
  const double de = delta == 0.0 ? 0.01 * rtol : delta;
  double h = 0.9 * sqrt(rtol / de);
  h = jmin(jmax(h, p.dt_var_min), p.dt_var_max);
  return jmin(jmax(dt * h, p.dt_min), p.dt_max);
}

struct ElemIn {
  const double *sol, *delta, *ymix, *fix_y;
  const uint8_t* fix_mask;
  double pos_cut, nega_cut, mtol;
};

// Fixed-species override and clip of one element (outer_loop.py:733-739,
// 209-213). Returns the clipped value; v_in / d_in are the overridden inputs.
__device__ __forceinline__ double clip_elem(const ElemIn& E, int64_t e, double& v_in, double& d_in) {
  double v = E.sol[e];
  double d = E.delta[e];
  if (E.fix_mask && E.fix_mask[e]) {
    v = E.fix_y[e];
    d = 0.0;
  }
  v_in = v;
  d_in = d;
  double c = (v < E.pos_cut && v >= E.nega_cut) ? 0.0 : v;
  if (E.ymix[e] < E.mtol && c < 0.0) c = 0.0;
  return c;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__global__ void __launch_bounds__(BODY_THREADS)
loop_body_kernel(Batch B, VbLoopParams p, const uint8_t* __restrict__ gas, const double* __restrict__ compo,
                 const double* __restrict__ atom_ini, const double* __restrict__ atm, ElemIn E,
                 double* y, double* y_prev, double* ymix,  // may alias one another (y == y_prev)
                 double* __restrict__ atom_loss, double* __restrict__ atom_loss_prev, double* __restrict__ dtp,
                 VbLoopScalars* __restrict__ st, const VbConvState* __restrict__ conv, double* __restrict__ pre_y,
                 double* __restrict__ pre_ymix, double* __restrict__ pre_td) {
  extern __shared__ double ys[];  // [2][nz]: ysum of the clipped and of the rebalanced state
  __shared__ double red[BODY_WARPS][4 + 2 * VB_LOOP_MAX_ATOMS];
  __shared__ int flags_s[BODY_WARPS][2];
  __shared__ int decision;  // 0 reject, 1 accept, 2 force-accept

  const int b = blockIdx.x;
  if (conv && conv[b].done) return;  // stopped by the loop condition: frozen
  const Geo g = geo_of(B, b);
  const int ni = B.ni, nz = g.nz, na = p.n_atoms;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t o = g.z0 * ni;
  const double* M = atm + g.atm + atm_offsets(nz, ni).M;
  const bool hydro = (p.flags & VB_LOOP_HYDRO_PARTIAL) != 0;
  const bool bot0 = (p.flags & VB_LOOP_ZERO_BOT_ROW) != 0;
  ElemIn Eb = E;
  Eb.sol += o;
  Eb.delta += o;
  Eb.ymix += o;
  if (Eb.fix_mask) {
    Eb.fix_mask += o;
    Eb.fix_y += o;
  }
  double* ysc = ys;
  double* ysb = ys + nz;

  // ---- phase A: clip, error norm, flags, clipped mass, ysums, atom sums
  double dmax = 0.0, small = 0.0, nega = 0.0;
  int notnonneg = 0, anyneg = 0;
  double pn[VB_LOOP_MAX_ATOMS], pb[VB_LOOP_MAX_ATOMS];
#pragma unroll
  for (int a = 0; a < VB_LOOP_MAX_ATOMS; ++a) pn[a] = pb[a] = 0.0;
  for (int j = warp; j < nz; j += BODY_WARPS) {
    double cv[4];
    double gs = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = lane + 32 * q;
      cv[q] = 0.0;
      if (i < ni) {
        const int64_t e = (int64_t)j * ni + i;
        double v, d;
        const double c = clip_elem(Eb, e, v, d);
        small += (v < p.pos_cut && v >= 0.0) ? fabs(v) : 0.0;
        nega += (v > p.nega_cut && v <= 0.0) ? fabs(v) : 0.0;
        double m = (Eb.ymix[e] < p.mtol) ? 0.0 : d;
        if (c < p.atol) m = 0.0;
        if (bot0 && j == 0) m = 0.0;
        if ((p.cond_zero_bits[i >> 5] >> (i & 31)) & 1u) m = 0.0;
        const double ratio = (c > 0.0) ? m / fmax(fabs(c), 1e-300) : 0.0;
        dmax = jmax(dmax, ratio);
        notnonneg |= !(c >= 0.0);
        anyneg |= (c < 0.0);
        if (!gas || gas[i]) gs += c;
        cv[q] = c;
      }
    }
    const double ysum_c = warp_sum(gs);
    double bs = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = lane + 32 * q;
      if (i < ni) {
        const bool gi = !gas || gas[i];
        const double bv = (hydro && !gi) ? cv[q] : M[j] * (cv[q] / ysum_c);
        if (gi) bs += bv;
#pragma unroll
        for (int a = 0; a < VB_LOOP_MAX_ATOMS; ++a) {
          if (a < na) {
            const double w = compo[i * na + a];
            pn[a] += w * cv[q];
            pb[a] += w * bv;
          }
        }
      }
    }
    const double ysum_b = warp_sum(bs);
    if (lane == 0) {
      ysc[j] = ysum_c;
      ysb[j] = ysum_b;
    }
  }
  // block reductions (fixed order: lanes by xor tree, then warps in index order)
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    dmax = jmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
    small += __shfl_xor_sync(0xffffffffu, small, off);
    nega += __shfl_xor_sync(0xffffffffu, nega, off);
  }
#pragma unroll
  for (int a = 0; a < VB_LOOP_MAX_ATOMS; ++a) {
    if (a < na) {
      pn[a] = warp_sum(pn[a]);
      pb[a] = warp_sum(pb[a]);
    }
  }
  notnonneg = __any_sync(0xffffffffu, notnonneg);
  anyneg = __any_sync(0xffffffffu, anyneg);
  if (lane == 0) {
    red[warp][0] = dmax;
    red[warp][1] = small;
    red[warp][2] = nega;
    for (int a = 0; a < na; ++a) {
      red[warp][4 + a] = pn[a];
      red[warp][4 + VB_LOOP_MAX_ATOMS + a] = pb[a];
    }
    flags_s[warp][0] = notnonneg;
    flags_s[warp][1] = anyneg;
  }
  __syncthreads();

  // ---- decision (thread 0)
  if (threadIdx.x == 0) {
    double delta = red[0][0], sm = red[0][1], ng = red[0][2];
    int nn = flags_s[0][0], an = flags_s[0][1];
    for (int w = 1; w < BODY_WARPS; ++w) {
      delta = jmax(delta, red[w][0]);
      sm += red[w][1];
      ng += red[w][2];
      nn |= flags_s[w][0];
      an |= flags_s[w][1];
    }
    VbLoopScalars s = st[b];
    const double dt = dtp[b];
    if (pre_td) {   // the attempt's start time and step, which condensation reads
      pre_td[2 * (int64_t)b] = s.t;
      pre_td[2 * (int64_t)b + 1] = dt;
    }
    double* alb = atom_loss + (int64_t)b * na;
    double* alp = atom_loss_prev + (int64_t)b * na;
    const double* ini = atom_ini + (int64_t)b * na;
    double loss_diff = 0.0, max_loss = 0.0;
    double al_new[VB_LOOP_MAX_ATOMS], al_bal[VB_LOOP_MAX_ATOMS];
    for (int a = 0; a < na; ++a) {
      double sn = red[0][4 + a], sb = red[0][4 + VB_LOOP_MAX_ATOMS + a];
      for (int w = 1; w < BODY_WARPS; ++w) {
        sn += red[w][4 + a];
        sb += red[w][4 + VB_LOOP_MAX_ATOMS + a];
      }
      al_new[a] = (sn - ini[a]) / ini[a];
      al_bal[a] = (sb - ini[a]) / ini[a];
      loss_diff = a == 0 ? fabs(al_new[a] - alp[a]) : jmax(loss_diff, fabs(al_new[a] - alp[a]));
      max_loss = a == 0 ? fabs(al_new[a]) : jmax(max_loss, fabs(al_new[a]));
    }
    double rtol = s.rtol;
    const bool accept = !nn && (loss_diff < p.loss_eps) && (delta <= rtol);
    const double next_reject = dt * p.dt_var_min;
    const bool force = ((next_reject < p.dt_min) || (s.retry_count >= p.batch_max_retries)) && !accept;
    const bool take = accept || force;
    const bool too_big = delta > rtol;
    const int acc0 = s.accept_count;
    if (take) s.t = s.t + (force ? p.dt_min : dt);
    if (force) {
      for (int a = 0; a < na; ++a) alb[a] = alp[a];
    } else if (accept) {
      for (int a = 0; a < na; ++a) alb[a] = al_bal[a];
    }
    if (take) {
      for (int a = 0; a < na; ++a) alp[a] = alb[a];
      s.accept_count += 1;
      s.retry_count = 0;
      s.small_y = s.small_y + sm;
      s.nega_y = s.nega_y + ng;
    } else {
      s.retry_count += 1;
      if (too_big) s.delta_count += 1;
      else if (an) s.nega_count += 1;
      else s.loss_count += 1;
    }
    double lc = s.loss_criteria;
    if ((p.flags & VB_LOOP_ADAPT_RTOL) && take) {
      if (acc0 % p.adapt_rtol_dec_period == 0 && max_loss >= lc) {
        rtol = jmax(rtol * p.adapt_rtol_dec, p.rtol_min);
        lc = lc * p.adapt_rtol_loss_mul;
      }
      if (acc0 % p.adapt_rtol_inc_period == 0 && acc0 > 0 && max_loss < p.adapt_rtol_inc_loss_thresh)
        rtol = jmin(rtol * p.adapt_rtol_inc, p.rtol_max);
    }
    const double dt_norm = step_size(dt, delta, rtol, p);
    const double dt_force = step_size(p.dt_min, delta, rtol, p);
    dtp[b] = force ? dt_force : (accept ? dt_norm : next_reject);
    s.rtol = rtol;
    s.loss_criteria = lc;
    s.delta = delta;
    s.last_decision = force ? 2 : (accept ? 1 : 0);
    st[b] = s;
    decision = s.last_decision;
  }
  __syncthreads();

  // ---- phase B: next y / y_prev / ymix
  const int dec = decision;
  double* yb = y + o;
  double* ypb = y_prev + o;
  double* xb = ymix + o;
  // the attempt's clipped state (sol_clip, ymix_new of outer_loop.py:740),
  // which the atmosphere refresh of an accepted or force-accepted attempt
  // reads (outer_loop.py:818-826); written before the state is overwritten
  if (pre_y && dec != 0) {
    for (int j = warp; j < nz; j += BODY_WARPS) {
      const double sc = ysc[j];
      for (int i = lane; i < ni; i += 32) {
        const int64_t e = (int64_t)j * ni + i;
        double v, d;
        const double c = clip_elem(Eb, e, v, d);
        pre_y[o + e] = c;
        pre_ymix[o + e] = c / sc;
      }
    }
  }
  if (dec == 1) {
    for (int j = warp; j < nz; j += BODY_WARPS) {
      const double sc = ysc[j], sb = ysb[j], Mj = M[j];
      for (int i = lane; i < ni; i += 32) {
        const int64_t e = (int64_t)j * ni + i;
        double v, d;
        const double c = clip_elem(Eb, e, v, d);
        const bool gi = !gas || gas[i];
        const double bv = (hydro && !gi) ? c : Mj * (c / sc);
        yb[e] = bv;
        ypb[e] = bv;
        xb[e] = bv / sb;
      }
    }
  } else {
    const int n = nz * ni;
    for (int e = threadIdx.x; e < n; e += BODY_THREADS) {
      double v = ypb[e];
      if (dec == 2) {
        v = v < 0.0 ? 0.0 : v;
        ypb[e] = v;
      }
      yb[e] = v;
    }
  }
}

cudaError_t launch_loop_body(const Batch& B, const VbLoopParams& p, const uint8_t* gas, const double* compo,
                             const double* atom_ini, const double* atm, const uint8_t* fix_mask,
                             const double* fix_y, const double* sol, const double* delta, double* y,
                             double* y_prev, double* ymix, double* atom_loss, double* atom_loss_prev,
                             double* dt, VbLoopScalars* st, const VbConvState* conv, double* pre_y,
                             double* pre_ymix, double* pre_td, cudaStream_t stream) {
  ElemIn E;
  E.sol = sol;
  E.delta = delta;
  E.ymix = ymix;
  E.fix_y = fix_y;
  E.fix_mask = fix_mask;
  E.pos_cut = p.pos_cut;
  E.nega_cut = p.nega_cut;
  E.mtol = p.mtol;
  const size_t smem = 2 * (size_t)B.nz * sizeof(double);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(loop_body_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  loop_body_kernel<<<B.count, BODY_THREADS, smem, stream>>>(B, p, gas, compo, atom_ini, atm, E, y, y_prev, ymix,
                                                            atom_loss, atom_loss_prev, dt, st, conv, pre_y,
                                                            pre_ymix, pre_td);
  return cudaGetLastError();
}

// Convergence after the body (one CTA per atmosphere). Ring slot
// max(accept_count - 1, 0) % conv_step takes (y, t) (outer_loop.py:918-928);
// the lookback entry is the first slot, the one just written excluded, whose
// t is nearest t * st_factor (_conv_jax, :633-670); longdy is the largest
// |y - y_old| / n_0 / ymix over the entries with ymix >= mtol_conv,
// y >= atol and the species not ignored, longdydt = longdy / (t - t_old);
// both kept only after an accepted (or force-accepted) step, with the stall
// counter restarting on a 5 % drop below the lowest longdy seen (:944-989);
// photo-frequency switch (:1040-1050); cond_fn (:672-713) -> done.
__global__ void __launch_bounds__(BODY_THREADS)
loop_conv_kernel(Batch B, VbConvParams p, const double* __restrict__ atm, const double* __restrict__ slope_min,
                 const uint8_t* __restrict__ ignore, const double* __restrict__ y, const double* __restrict__ ymix,
                 const VbLoopScalars* __restrict__ st, double* __restrict__ ring_y, double* __restrict__ ring_t,
                 VbConvState* __restrict__ conv, int32_t* __restrict__ photo_due) {
  __shared__ double red[BODY_WARPS];
  __shared__ int k_s;
  const int b = blockIdx.x;
  if (conv[b].done) {
    if (photo_due && threadIdx.x == 0) photo_due[b] = 0;
    return;
  }
  const Geo g = geo_of(B, b);
  const int ni = B.ni, nz = g.nz, n = nz * ni;
  const int64_t o = g.z0 * ni;
  const VbLoopScalars s = st[b];
  const int cs = p.conv_step;
  const int idx = (s.accept_count > 0 ? s.accept_count - 1 : 0) % cs;
  double* ry = ring_y + o * cs;
  double* rt = ring_t + (int64_t)b * cs;
  const double* M = atm + g.atm + atm_offsets(nz, ni).M;
  const double* yb = y + o;
  const double* xb = ymix + o;
  if (threadIdx.x == 0) {
    rt[idx] = s.t;
    const double target = s.t * p.st_factor;
    int k = -1;
    double best = 0.0;
    for (int q = 0; q < cs; ++q) {
      const double dq = q == idx ? INFINITY : fabs(rt[q] - target);
      if (k < 0 || dq < best) {
        k = q;
        best = dq;
      }
    }
    k_s = k;
  }
  __syncthreads();
  const int k = k_s;
  const double* yo = ry + (int64_t)k * n;
  double mx = 0.0;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int j = e / ni, i = e - j * ni;
    const double yv = yb[e], xv = xb[e];
    double la = fabs((yv - yo[e]) / M[j]);
    if (xv < p.mtol_conv) la = 0.0;
    if (yv < p.atol) la = 0.0;
    if (ignore && ignore[i]) la = 0.0;
    const double ratio = xv > 0.0 ? la / fmax(xv, 1e-300) : 0.0;
    mx = jmax(mx, ratio);
  }
  __syncthreads();  // every thread has read the lookback entry before the slot is rewritten
  double* slot = ry + (int64_t)idx * n;
  for (int e = threadIdx.x; e < n; e += blockDim.x) slot[e] = yb[e];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = jmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double ld_new = red[0];
    for (int w = 1; w < BODY_WARPS; ++w) ld_new = jmax(ld_new, red[w]);
    const double ldt_new = ld_new / fmax(s.t - rt[k], 1e-300);
    VbConvState c = conv[b];
    const bool take = s.last_decision != 0;
    if (take) {
      c.longdy = ld_new;
      c.longdydt = ldt_new;
    }
    const bool drop = take && (c.longdy < c.longdy_seen_min * 0.95);
    if (drop) {
      c.longdy_seen_min = c.longdy;
      c.count_since_new_min = 0;
    } else if (take) {
      c.count_since_new_min += 1;
    }
    if (p.use_photo && !c.is_final_photo_frq && c.longdy < p.photo_switch_longdy &&
        c.longdydt < p.photo_switch_longdydt) {
      c.update_photo_frq = p.final_update_photo_frq;
      c.is_final_photo_frq = 1;
    }
    const bool too_long = s.t > p.runtime;
    const bool too_many = s.accept_count > p.count_max;
    bool converged = ((c.longdy < p.yconv_cri) && (c.longdydt < p.slope_cri)) ||
                     ((c.longdy < p.yconv_min) && (c.longdydt < slope_min[b]));
    converged = converged && (c.aflux_change < p.flux_cri);
    const bool stalled = (c.count_since_new_min > p.conv_stall_window) && (c.longdy_seen_min < p.yconv_min) &&
                         (c.longdy < p.yconv_min) && (c.aflux_change < p.flux_cri);
    const bool ready = (s.t > p.trun_min) && (s.accept_count > p.count_min);
    c.done = (too_long || too_many || (ready && (converged || stalled))) ? 1 : 0;
    conv[b] = c;
    if (photo_due)
      photo_due[b] = (!c.done && p.use_photo && c.update_photo_frq > 0 && s.retry_count == 0 &&
                      s.accept_count % c.update_photo_frq == 0)
                         ? 1
                         : 0;
  }
}

cudaError_t launch_loop_conv(const Batch& B, const VbConvParams& p, const double* atm, const double* slope_min,
                             const uint8_t* ignore, const double* y, const double* ymix, const VbLoopScalars* st,
                             double* ring_y, double* ring_t, VbConvState* conv, int32_t* photo_due,
                             cudaStream_t stream) {
  loop_conv_kernel<<<B.count, BODY_THREADS, 0, stream>>>(B, p, atm, slope_min, ignore, y, ymix, st, ring_y, ring_t,
                                                         conv, photo_due);
  return cudaGetLastError();
}

}  // namespace vb
