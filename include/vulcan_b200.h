/*
 * vulcan_b200.h - C-ABI of the B200-native Ros2 step and block-Thomas solve.
 *
 * Every entry point takes plain pointers and sizes. Array arguments marked
 * "device" are caller-owned device memory; all compute entry points are
 * stream-ordered and asynchronous (no host synchronisation, no allocation).
 * Only vb_net_create / vb_net_destroy allocate (set-up time).
 *
 * Return value of every function: 0 on success, otherwise a VB_ERR_* code
 * (vb_last_error() gives a message). Per-atmosphere numerical status words
 * (VB_STATUS_*) are written to a caller-provided device int32 array.
 *
 * Layouts (FP64 unless stated; "batch" atmospheres, uniform shapes or ragged
 * layer counts given by the prefix sums `zoff`):
 *   y, sol, delta     [B][nz][ni]            (species contiguous)
 *   k                 [B][nr+1][nz]          (layers contiguous; row 0 unused)
 *   dt                [B]
 *   fix_mask          [B][nz][ni] uint8 or NULL
 *   atm blob          [B][VB_ATM_DOUBLES(nz, ni)]  (see vb_atm_offsets)
 *   workspace         vb_ros2_workspace_bytes(...)
 * With ragged batches (zoff != NULL, zoff[B] = total layers) atmosphere b has
 * nz_b = zoff[b+1]-zoff[b] layers and its arrays start at zoff[b]*ni (y),
 * zoff[b]*(nr+1) (k), vb_atm_offset(...) (atm) in the packed buffers.
 */
#ifndef VULCAN_B200_H
#define VULCAN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VB_OK 0
#define VB_ERR_ARG 1        /* invalid argument (size, pointer, ni too large) */
#define VB_ERR_CUDA 2       /* a CUDA runtime call failed */
#define VB_ERR_ALLOC 3      /* set-up allocation failed */

#define VB_STATUS_OK 0
#define VB_STATUS_ZERO_PIVOT 1     /* an exactly zero pivot in a diagonal block */
#define VB_STATUS_NONFINITE 2      /* a non-finite value in the result */
#define VB_STATUS_REFINE_STALL 4   /* mixed path: refinement stalled, FP64 refactor used */
#define VB_STATUS_WATCHDOG 8       /* a bounded wait gave up (kernel returned early) */

/* Transport switches (reference jax_step.py:46-49 AtmStatic flags). */
#define VB_USE_VM_MOL 1
#define VB_USE_SETTLING 2
#define VB_USE_TOPFLUX 4
#define VB_USE_BOTFLUX 8

/* Largest species count the kernels accept. */
#define VB_MAX_NI 128

/* Atmosphere blob: per-atmosphere packing of the reference AtmStatic
 * (jax_step.py:26-49). Per-layer arrays take nz slots (interface arrays use
 * the first nz-1). Field order, in doubles from the atmosphere's base:
 *   Kzz[nz] dzi[nz] vz[nz] Hpi[nz] Ti[nz] Tco[nz] g[nz] M[nz]
 *   Dzz[nz][ni] vm[nz][ni] vs[nz][ni]
 *   ms[ni] alpha[ni] top_flux[ni] bot_flux[ni] bot_vdep[ni] gas_mask[ni] (0/1)  */
#define VB_ATM_DOUBLES(nz, ni) ((size_t)(nz) * (8 + 3 * (size_t)(ni)) + 6 * (size_t)(ni))

typedef struct VbNet VbNet;  /* opaque, device-resident network tables */

const char* vb_last_error(void);
int vb_version(void);

/* Network tables (reference chem.py:28-80 NetworkArrays, from network.py:197-491).
 * Host arrays: reactant_idx/product_idx [nr+1][max_terms] (padding index = ni),
 * reactant/product_stoich [nr+1][max_terms], is_three_body [nr+1].
 * Builds the gather tables of the RHS and Jacobian scatters on the host and
 * uploads them (the only allocating call). */
int vb_net_create(int ni, int nr, int max_terms,
                  const int64_t* reactant_idx, const int64_t* product_idx,
                  const double* reactant_stoich, const double* product_stoich,
                  const uint8_t* is_three_body, VbNet** out);
int vb_net_destroy(VbNet* net);
/* Launch shapes of the steps run with a network (no counterpart in the
 * reference, whose XLA compiler picks its own): set by the project's
 * autotuner (jax-vulcan_b200/autotune.py), which times the candidates on the
 * device per network and batch; 0 in a field = the automatic choice.
 *   factor_kernel: 1 blocked Gauss-Jordan on the tensor cores, 2 scalar
 *                  Gauss-Jordan, 3 scalar Gauss-Jordan pipelined per column
 *                  panel, 4 scalar Gauss-Jordan with two atmospheres per CTA
 *                  (uniform batches of 65-72 species; else as 2) (0: the
 *                  process default, vb_set_factor_kernel)
 *   factor_ctas:   CTAs per SM of the factor, 1 or 2 (honoured for 65-72
 *                  species, the shape with both variants compiled)
 *   sweep_stages:  depth of the sweeps' bulk-copy ring, 1..3 (lowered when
 *                  the ring does not fit in shared memory)
 *   streams:       2 = vb_ros2_step runs the two halves of a uniform batch
 *                  on the caller's stream and a second stream of the
 *                  library's (created on first use, one per device; forked
 *                  and joined with events, so the call stays stream-ordered
 *                  on the caller's stream), so one half's assembly overlaps
 *                  the other half's factor; 0 or 1 = one stream
 *   stage1_layers: layers per CTA of the stage-1 and stage-2 assembly, 1 or
 *                  2 (two share every gather-table word and rate-constant
 *                  sector; 0 = the default, 1) */
typedef struct VbTuning {
  int32_t factor_kernel, factor_ctas, sweep_stages, streams, stage1_layers, reserved;
} VbTuning;
int vb_net_set_tuning(VbNet* net, const VbTuning* tuning);
int vb_net_get_tuning(const VbNet* net, VbTuning* tuning);
/* Device bytes held by a network. */
size_t vb_net_device_bytes(const VbNet* net);

/* Ros2 step (replaces reference jax_step.py:249-315 jax_ros2_step, vmapped over
 * a batch). Inputs y, k, dt, atm, fix_mask (nullable); outputs sol, delta,
 * status[B]. zoff: NULL for a uniform batch of `nz` layers, else device int64
 * [B+1] prefix sums (then nz is the maximum layer count). */
size_t vb_ros2_workspace_bytes(int batch, int nz, int ni, const int64_t* zoff_host);
/* Optional extra workspace of vb_ros2_step (no reference counterpart): with
 * workspace_bytes >= the 256-byte-aligned vb_ros2_workspace_bytes(batch, nz,
 * ni, NULL) + vb_ros2_assembly_bytes(net, batch, nz) (nz: the maximum layer
 * count of a ragged batch), the step assembles the stage-2 right-hand side
 * with one thread per layer (the rate of every reaction and layer staged in
 * that region, then every species sum formed from coalesced rows of layers)
 * instead of one CTA per layer; the results are identical. nr+1 doubles per
 * layer. */
size_t vb_ros2_assembly_bytes(const VbNet* net, int batch, int nz);
int vb_ros2_step(const VbNet* net, int batch, int nz, const int64_t* zoff,
                 const double* y, const double* k, const double* dt,
                 const double* atm, int32_t atm_flags, const uint8_t* fix_mask,
                 double* sol, double* delta, int32_t* status,
                 void* workspace, size_t workspace_bytes, void* stream);

/* Mixed-precision Ros2 step: the same inputs, outputs and FP64 interface as
 * vb_ros2_step, with the demotion inside. The LHS blocks are assembled in
 * FP64 (kept for the residual); each Schur-updated block is row-equilibrated
 * (exact powers of two) and inverted in FP32 by the process's factor kernel
 * (vb_set_factor_kernel: scalar Gauss-Jordan by default; the blocked kernel
 * runs its rank-8 trailing updates on the TF32 tensor cores, each operand
 * split into a TF32 head and tail, three products); each stage solve
 * LHS k = rhs (jax_step.py:300-311) starts from the FP32 factors and is
 * refined in FP64 on the full block-tridiagonal system (r = rhs - LHS k from
 * the FP64 blocks, k += M~^{-1} r) until max|correction| <= tol * max|k|, at
 * most max_refine passes; atmospheres whose refinement stalls (or whose FP32
 * factor meets a zero pivot or a non-finite value) are refactored in FP64
 * and solved directly, with VB_STATUS_REFINE_STALL. sol and delta are formed
 * in FP64 from the refined stages. passes [B] (nullable): solve and
 * refinement passes run per atmosphere over both stages. ni <= 96. The
 * workspace holds the FP64 step workspace, the FP32 inverses and row scales,
 * and per-atmosphere state (vb_ros2_mixed_workspace_bytes; a ragged batch
 * sizes it with zoff_host = NULL and nz = its maximum layer count). As with
 * vb_ros2_step, a workspace of at least the 256-byte-aligned
 * vb_ros2_mixed_workspace_bytes + vb_ros2_assembly_bytes(net, batch, nz)
 * bytes selects the thread-per-layer stage 2 (identical results). */
size_t vb_ros2_mixed_workspace_bytes(int batch, int nz, int ni, const int64_t* zoff_host);
int vb_ros2_step_mixed(const VbNet* net, int batch, int nz, const int64_t* zoff,
                       const double* y, const double* k, const double* dt,
                       const double* atm, int32_t atm_flags, const uint8_t* fix_mask,
                       int max_refine, double tol, double* sol, double* delta, int32_t* status,
                       int32_t* passes, void* workspace, size_t workspace_bytes, void* stream);

/* Stage vectors of the last vb_ros2_step run on `workspace` (the reference's
 * k1 and k2 of jax_step.py:300-311, which jax_ros2_step keeps internal):
 * k1, k2 [B][nz][ni] (or packed by zoff), either may be NULL. For checking a
 * step's two block solves by their backward errors; same batch arguments as
 * the step. Also valid after vb_ros2_step_mixed (its workspace starts with
 * the same layout). */
int vb_ros2_stages(const VbNet* net, int batch, int nz, const int64_t* zoff, const void* workspace,
                   double* k1, double* k2, void* stream);

/* Failure-detection testing: every bulk copy of the factor and sweep kernels
 * is awaited with a bounded poll loop; a wait that runs out sets
 * VB_STATUS_WATCHDOG for its atmosphere, drains the copies still in flight
 * (with the full limit) and returns early. vb_set_wait_limit sets the poll
 * limit of that first wait for later launches from this process (0: give up
 * at once); polls < 0 restores the default (2^22). No counterpart in the
 * reference (its solver has no waits). */
int vb_set_wait_limit(long long polls);
/* Poll limit of every wait between the warps of the pipelined factor
 * (vb_set_factor_kernel(2), VbTuning.factor_kernel 3) for later launches from
 * this process: a warp that gives up stops every other warp's wait, the
 * atmosphere gets VB_STATUS_WATCHDOG and its factor returns after draining
 * the prefetch in flight; polls < 0 restores the default (2^22). A test hook
 * with no counterpart in the reference. */
int vb_set_pipeline_wait_limit(long long polls);

/* FP64 block-factor kernel of the step, the block solver and the adjoint, for
 * later launches from this process (a network's VbTuning.factor_kernel
 * overrides it for that network): 0 = blocked Gauss-Jordan, one warp per
 * 8-column panel, the panel's pivot steps inside the warp and the rank-8
 * trailing updates on the FP64 tensor cores (mma.sync m8n8k4); 1 (default) =
 * scalar Gauss-Jordan, one block barrier per pivot step; 2 = the same scalar
 * elimination pipelined: the warp owning a column panel runs its pivot steps
 * back to back and publishes each (pivot row, multipliers) through a
 * shared-memory ring signalled by mbarriers, the other warps apply the steps
 * as they arrive (bounded waits; no block barrier per step); 3 = the scalar
 * elimination with two atmospheres per CTA, their pivot chains interleaved
 * in the same warps under one barrier per step (FP64 factor of uniform
 * batches of 65-72 species; the scalar kernel elsewhere). All replace the
 * reference's lu_factor + lu_solve(LU, I) pair (solver.py:46-48). */
int vb_set_factor_kernel(int variant);

/* Chemistry (reference chem.py:83-131 chem_rhs and chem.py:144-214
 * chem_jac_analytical, vmapped over layers and a uniform batch):
 * y [B][nz][ni], M [B][nz], k [B][nr+1][nz] -> dydt [B][nz][ni], jac [B][nz][ni][ni]. */
int vb_chem_rhs(const VbNet* net, int batch, int nz, const double* y, const double* M,
                const double* k, double* dydt, void* stream);
int vb_chem_jac(const VbNet* net, int batch, int nz, const double* y, const double* M,
                const double* k, double* jac, void* stream);

/* Diffusion (reference jax_step.py:67-246: compute_diff_grav,
 * _build_diff_coeffs_jax, _apply_diffusion_jax) for a uniform batch:
 * y [B][nz][ni], atm blob -> diff [B][nz][ni] (BC fluxes included) and the
 * block-Thomas diagonal terms diag_d [B][nz][ni] (bot_vdep included),
 * sup_d [B][nz-1][ni], sub_d [B][nz-1][ni] (NOT negated). */
int vb_diffusion(int batch, int nz, int ni, const double* y, const double* atm, int32_t atm_flags,
                 double* diff, double* diag_d, double* sup_d, double* sub_d, void* stream);

/* Block-tridiagonal Thomas with dense diagonal blocks and diagonal
 * off-diagonal blocks (reference solver.py:33-126), for a uniform batch.
 *   vb_bt_factor:  diag [B][nz][ni][ni], sup_d, sub_d [B][nz-1][ni] (the
 *                  off-diagonal blocks as passed to the reference solver) ->
 *                  factors (opaque, vb_bt_factor_bytes) + status.
 *   vb_bt_solve:   factors + rhs [B][nz][ni] -> x [B][nz][ni].
 *   vb_bt_solve_T: solves the transposed system (for the adjoint,
 *                  reference steady_state_grad.py:214-219): x = A^-T rhs. */
size_t vb_bt_factor_bytes(int batch, int nz, int ni);
int vb_bt_factor(int batch, int nz, int ni, const double* diag, const double* sup_d,
                 const double* sub_d, void* factors, int32_t* status, void* stream);
int vb_bt_solve(int batch, int nz, int ni, const void* factors, const double* rhs, double* x,
                void* stream);
int vb_bt_solve_T(int batch, int nz, int ni, const void* factors, const double* rhs, double* x,
                  void* stream);

/* Mixed-precision block solve (the solver of reference solver.py:33-112 with
 * the demotion inside, same FP64 interface): the diagonal blocks are factored
 * and inverted in FP32 (up to 96 species with every row of each Schur-updated
 * block first scaled by a power of two to magnitude [1, 2), the inverse
 * applied as X diag(r)), the solution is refined in FP64 on the full
 * block-tridiagonal system (r = rhs - M x from the FP64 blocks, x += M~^{-1} r
 * with the FP32 inverses) until max|correction| <= tol * max|x|, at most
 * max_refine passes after the first solve. Atmospheres whose refinement
 * stalls are refactored and solved in FP64 and get VB_STATUS_REFINE_STALL.
 *   vb_bt_mixed_bytes:  size of the factors buffer (FP64 blocks, FP32 and FP64
 *                       inverses, per-atmosphere state).
 *   vb_bt_factor_mixed: diag, sup_d, sub_d as vb_bt_factor -> factors, status.
 *   vb_bt_solve_mixed:  rhs -> x (must not alias rhs); status |= stall bits;
 *                       passes [B] (nullable): solve + refinement passes run. */
size_t vb_bt_mixed_bytes(int batch, int nz, int ni);
int vb_bt_factor_mixed(int batch, int nz, int ni, const double* diag, const double* sup_d,
                       const double* sub_d, void* factors, int32_t* status, void* stream);
int vb_bt_solve_mixed(int batch, int nz, int ni, void* factors, const double* rhs, double* x,
                      int max_refine, double tol, int32_t* status, int32_t* passes, void* stream);

/* Steady-state residual f(y) = chem_rhs + diffusion (reference
 * steady_state_grad.py:116-130) of a (possibly ragged) batch -> f [B][nz][ni]. */
int vb_residual(const VbNet* net, int batch, int nz, const int64_t* zoff, const double* y, const double* k,
                const double* atm, int32_t atm_flags, double* f, void* stream);

/* Implicit steady-state adjoint (reference steady_state_grad.py:153-233,
 * 284-330): assembles J_y = df/dy at y_star, solves J_y^T lambda = v with the
 * block-Thomas factors (transposed sweeps), and writes the cotangents
 * -lambda . df/dtheta (each output nullable): g_k [B][nr+1][nz] (the k_arr
 * leaf), g_M [B][nz], g_Kzz [B][nz] (interfaces 0..nz-2; packed by layers
 * like y for ragged batches),
 * g_top, g_bot, g_vdep [B][ni]; lambda [B][nz][ni] if non-NULL.
 * Uses the Ros2 workspace (vb_ros2_workspace_bytes). */
int vb_adjoint(const VbNet* net, int batch, int nz, const int64_t* zoff, const double* y_star, const double* k,
               const double* atm, int32_t atm_flags, const double* v, double* lambda, double* g_k, double* g_M,
               double* g_Kzz, double* g_top, double* g_bot, double* g_vdep, int32_t* status, void* workspace,
               size_t workspace_bytes, void* stream);

/* Loop body of the adaptive runner (reference outer_loop.py:715-1100, the
 * decision part of body_fn): given a Ros2 step's sol / delta_arr, applies the
 * fixed-species override, clip (:196-224), atom loss (:171-178), error norm
 * (:227-250), accept / force-accept / reject (:745-768), hydrostatic
 * rebalance (:844-853), next state (:899-917), counters (:1062-1066),
 * adaptive rtol (:990-1020) and the next dt (:181-193, :1022-1031), per
 * atmosphere, on the device. Photo, condensation, atmosphere refresh, ion
 * balance and bottom pins are not part of it; the convergence ring and the
 * loop condition are vb_loop_converge. */
#define VB_LOOP_MAX_ATOMS 16
#define VB_LOOP_HYDRO_PARTIAL 1  /* rebalance gas species only (use_condense) */
#define VB_LOOP_ZERO_BOT_ROW 2   /* drop the bottom layer from the error norm */
#define VB_LOOP_ADAPT_RTOL 4     /* adaptive rtol */
typedef struct VbLoopParams {
  int32_t n_atoms;               /* 1..VB_LOOP_MAX_ATOMS */
  int32_t batch_max_retries;
  int32_t flags;                 /* VB_LOOP_* */
  int32_t adapt_rtol_dec_period, adapt_rtol_inc_period;
  int32_t reserved;
  /* species whose delta the error norm drops in every layer (bit i % 32 of
   * word i / 32): the reference's condense_zero_mask, condense_sp + non_gas_sp
   * when use_condense is on (outer_loop.py:244, :1380-1386); all zero otherwise */
  uint32_t cond_zero_bits[4];
  double loss_eps, pos_cut, nega_cut, mtol, atol;
  double dt_var_min, dt_var_max, dt_min, dt_max;
  double rtol_min, rtol_max, adapt_rtol_dec, adapt_rtol_inc, adapt_rtol_loss_mul, adapt_rtol_inc_loss_thresh;
} VbLoopParams;
/* Per-atmosphere scalars of the loop carry (JaxIntegState fields of the same
 * names), device memory, updated in place; dt is a separate [B] array so the
 * same buffer feeds vb_ros2_step. last_decision: 0 reject, 1 accept,
 * 2 force-accept. */
typedef struct VbLoopScalars {
  double t, delta, small_y, nega_y, rtol, loss_criteria;
  int32_t accept_count, retry_count, nega_count, loss_count, delta_count, last_decision;
} VbLoopScalars;
/* Convergence and termination knobs (reference _Statics, outer_loop.py:420-460;
 * defaults in vulcan_cfg). conv_step >= 2 is the ring length. */
typedef struct VbConvParams {
  int32_t conv_step, count_min, count_max, conv_stall_window;
  int32_t use_photo, final_update_photo_frq, reserved0, reserved1;
  double st_factor, mtol_conv, atol, yconv_cri, yconv_min, slope_cri, flux_cri, trun_min, runtime;
  double photo_switch_longdy, photo_switch_longdydt;
} VbConvParams;
/* Per-atmosphere convergence carry (JaxIntegState fields of the same names),
 * device memory, updated in place by vb_loop_converge. Start: longdy =
 * longdydt = 1, longdy_seen_min = +inf, count_since_new_min = 0, done = 0,
 * update_photo_frq = the initial photo frequency. aflux_change is written by
 * vb_photo_update. done = 1 once the loop condition stops the atmosphere;
 * vb_loop_body and vb_loop_converge then leave it alone. */
typedef struct VbConvState {
  double longdy, longdydt, longdy_seen_min, aflux_change;
  int32_t count_since_new_min, done, update_photo_frq, is_final_photo_frq;
} VbConvState;
/* Device arrays: gas_mask [ni] uint8 or NULL (non-gas species present: the
 * ysums of clip and mix run over gas species), compo [ni][n_atoms],
 * atom_ini [B][n_atoms], fix_mask [B][nz][ni] uint8 and fix_y [B][nz][ni]
 * (both NULL without fixed species), sol / delta_arr [B][nz][ni] (inputs;
 * must not alias the state), state: y, y_prev, ymix [B][nz][ni] (y may equal
 * y_prev), atom_loss, atom_loss_prev [B][n_atoms], dt [B], scalars [B]. The layer
 * densities n_0 are the atmosphere blob's M. zoff as in vb_ros2_step (nz is
 * then the maximum layer count). conv [B] (nullable): atmospheres whose record
 * has done set are skipped. pre_y, pre_ymix [B][nz][ni] (nullable, together):
 * for an accepted or force-accepted attempt, the attempt's clipped state
 * (sol_clip and ymix_new, outer_loop.py:740), the input of the atmosphere
 * refresh (vb_loop_refresh) and the condensation (vb_loop_condense). pre_td
 * [B][2] (nullable): the attempt's start time t and step dt. */
int vb_loop_body(int batch, int nz, int ni, const int64_t* zoff, const VbLoopParams* params,
                 const double* atm, const uint8_t* gas_mask, const double* compo, const double* atom_ini,
                 const uint8_t* fix_mask, const double* fix_y, const double* sol, const double* delta_arr,
                 double* y, double* y_prev, double* ymix, double* atom_loss, double* atom_loss_prev,
                 double* dt, VbLoopScalars* scalars, const VbConvState* conv, double* pre_y, double* pre_ymix,
                 double* pre_td, void* stream);

/* Convergence part of the adaptive runner, after vb_loop_body: writes (y, t)
 * into ring slot max(accept_count - 1, 0) % conv_step (outer_loop.py:918-928),
 * finds the ring entry nearest t * st_factor (the slot just written excluded),
 * computes longdy = max masked |y - y_old| / n_0 / ymix and longdydt =
 * longdy / (t - t_old) (_conv_jax, :633-670), keeps them only after an
 * accepted step, runs the stall counter (:944-989) and the photo-frequency
 * switch (:1040-1050), and evaluates cond_fn (:672-713) into conv[b].done.
 * Device arrays: slope_min [B] (cond_fn's slope floor), ignore_mask [ni]
 * uint8 or NULL (species left out of longdy), y, ymix [B][nz][ni],
 * scalars [B], ring_y [B][conv_step][nz][ni], ring_t [B][conv_step],
 * conv [B], photo_due [B] int32 or NULL (set to 1 where the next attempt
 * should run the photo branch: not done, use_photo, retry_count == 0 and
 * accept_count % update_photo_frq == 0, as outer_loop.py:716-724). With zoff,
 * atmosphere b's ring starts at zoff[b] * ni * conv_step. */
int vb_loop_converge(int batch, int nz, int ni, const int64_t* zoff, const VbConvParams* params, const double* atm,
                     const double* slope_min, const uint8_t* ignore_mask, const double* y, const double* ymix,
                     const VbLoopScalars* scalars, double* ring_y, double* ring_t, VbConvState* conv,
                     int32_t* photo_due, void* stream);

/* Cotangents of every transport leaf of the steady-state residual
 * (reference steady_state_grad.py:36-59 SteadyStateInputs leaves Kzz, Dzz,
 * dzi, vz, Hpi, Ti, Tco, g, ms, alpha, vm, vs, top_flux, bot_flux, bot_vdep;
 * the VJP of steady_state_grad.py:224-233): given lambda [B][nz][ni] (from
 * vb_adjoint), g_atm = -lambda . d diffusion / d leaf, written in the layout
 * of the atmosphere blob ([B][VB_ATM_DOUBLES(nz, ni)], same field order; the
 * M and gas-mask slots and the unused last slot of interface arrays are 0:
 * M's cotangent is vb_adjoint's g_M). With zoff the caller zeroes g_atm. */
int vb_adjoint_atm(int batch, int nz, int ni, const int64_t* zoff, const double* y_star, const double* atm,
                   int32_t atm_flags, const double* lambda, double* g_atm, void* stream);

/* Photochemistry (reference photo.py). Cross sections and branch tables are
 * device arrays shared by the batch, except the temperature-dependent tables
 * absp_T_cross [n_abs_T][nz][nbin] and cross_J_T [n_br_T][nz][nbin], which
 * advance by T_stride / T_stride_J doubles per atmosphere (0: shared). */
typedef struct VbPhoto {
  int32_t nbin, n_abs, n_abs_T, n_scat, n_br, n_br_T, din12, reserved;
  int64_t T_stride, T_stride_J;
  const int32_t* absp_idx;      /* [n_abs]   species of the T-independent absorbers */
  const int32_t* absp_T_idx;    /* [n_abs_T] species of the T-dependent absorbers */
  const int32_t* scat_idx;      /* [n_scat]  scattering species */
  const double* absp_cross;     /* [n_abs][nbin] */
  const double* absp_T_cross;   /* [n_abs_T][nz][nbin] */
  const double* scat_cross;     /* [n_scat][nbin] */
  const double* cross_J;        /* [n_br][nbin]   branch cross sections */
  const double* cross_J_T;      /* [n_br_T][nz][nbin] */
  const double* bins;           /* [nbin] wavelengths (nm) */
  const double* sflux_top;      /* [nbin] stellar flux at the top */
  const int32_t* br_re_idx;     /* [n_br]  k row of each branch */
  const int32_t* br_T_re_idx;   /* [n_br_T] */
  const uint8_t* br_active;     /* [n_br]  write the k row (reference remove_list) */
  const uint8_t* br_T_active;   /* [n_br_T] */
  double dbin1, dbin2, mu_zenith, edd, ag0, hc, f_diurnal;
} VbPhoto;

/* Optical depth (reference photo.py:84-123): y [B][nz][ni], dz [B][nz] ->
 * tau [B][nz+1][nbin] (tau[nz] = 0). */
int vb_photo_tau(int batch, int nz, int ni, const VbPhoto* photo, const double* y, const double* dz,
                 double* tau, void* stream);
/* Two-stream flux (reference photo.py:126-245): tau, ymix [B][nz][ni],
 * dflux_u_prev [B][nz+1][nbin] -> aflux [B][nz][nbin], sflux, dflux_d,
 * dflux_u [B][nz+1][nbin]. */
int vb_photo_flux(int batch, int nz, int ni, const VbPhoto* photo, const double* tau, const double* ymix,
                  const double* dflux_u_prev, double* aflux, double* sflux, double* dflux_d,
                  double* dflux_u, void* stream);
/* J-rates (reference photo.py:309-351) -> J_br [B][n_br][nz], J_br_T
 * [B][n_br_T][nz] (either nullable), and with k != NULL the photolysis rows
 * k[B][nr+1][nz] of active branches are set to J * f_diurnal
 * (photo.py:455-478). */
int vb_photo_j(int batch, int nz, int nr, const VbPhoto* photo, const double* aflux, double* J_br,
               double* J_br_T, double* k, void* stream);
/* The photo branch of the adaptive loop (reference outer_loop.py:283-350,
 * gated as outer_loop.py:716-724): tau -> flux -> J -> photolysis rows of k
 * for the atmospheres with due[b] != 0 (due NULL: all); the others are left
 * untouched. dflux_u [B][nz+1][nbin] holds the previous call's upward flux on
 * entry and the new one on return. With conv != NULL, conv[b].aflux_change of
 * each updated atmosphere becomes the largest |aflux_new - aflux_old| /
 * |aflux_new| over the entries with aflux_new > flux_atol (0 if none), where
 * aflux_old is what `aflux` held on entry. J_br / J_br_T nullable; k as
 * vb_ros2_step's [B][nr+1][nz]. */
int vb_photo_update(int batch, int nz, int ni, int nr, const VbPhoto* photo, const int32_t* due, const double* y,
                    const double* dz, const double* ymix, double* tau, double* aflux, double* sflux,
                    double* dflux_d, double* dflux_u, double* J_br, double* J_br_T, double* k, double flux_atol,
                    VbConvState* conv, void* stream);

/* Rate constants on the device (reference rates.py:61-208 and gibbs.py:41-150):
 * per layer, the forward constant of every forward row (modified Arrhenius
 * a T^n exp(-E/T); Lindemann k0 / (1 + k0 M / k_inf); the hardcoded Troe of
 * OH + CH3 + M -> CH3OH + M), the low-temperature caps, the reverse constant
 * k_f / K_eq with K_eq = exp(sum st g(reactants) - sum st g(products))
 * (k_B T / 1e6)^(dn) from NASA-9 g/RT, and the removal of listed rows.
 * code[i] of forward row i (odd): VB_RK_* kind | cap << 2 | VB_RC_* bits. */
#define VB_RK_NONE 0          /* left at zero (photo, ion, condensation, radiative, ...) */
#define VB_RK_ARRHENIUS 1
#define VB_RK_LINDEMANN 2
#define VB_RK_TROE_OH_CH3 3
#define VB_RCAP_CH3 1         /* H + CH3 + M -> CH4 + M, T <= 277.5 K */
#define VB_RCAP_C2H4 2        /* H + C2H4 + M -> C2H5 + M, T <= 300 K */
#define VB_RCAP_C2H5 3        /* H + C2H5 + M -> C2H6 + M, T <= 200 K */
#define VB_RC_THERMAL 16      /* K_eq from the Gibbs energies (else K_eq = 1) */
#define VB_RC_REVERSE 32      /* row i+1 is a reverse row (i+1 < stop_rev_indx); else it stays zero */
#define VB_RC_DROP_FWD 64     /* row i is removed (zeroed after the reverse fill) */
#define VB_RC_DROP_REV 128    /* row i+1 is removed */
#define VB_RATES_LOWT_CAPS 1  /* apply the low-temperature caps */
typedef struct VbRateTables {
  int32_t nr, ni, max_terms, reserved;
  const int32_t* code;        /* [nr+1] (forward rows used) */
  const double* par;          /* [nr+1][6]: a, n, E, a_inf, n_inf, E_inf */
  const double* nasa9;        /* [ni][2][10]: low-T (T < 1000 K) and high-T coefficients */
  const int32_t* r_idx;       /* [nr+1][max_terms] reactant species, padding ni */
  const int32_t* p_idx;       /* [nr+1][max_terms] product species, padding ni */
  const double* r_st;         /* [nr+1][max_terms] */
  const double* p_st;         /* [nr+1][max_terms] */
} VbRateTables;
/* T, M [B][nz] -> k [B][nr+1][nz] (row 0 zero); dkdT (nullable, same layout)
 * = dk/dT at fixed M, by dual numbers through the same formulas. */
int vb_rates(int batch, int nz, const VbRateTables* tables, const double* T, const double* M, int32_t flags,
             double* k, double* dkdT, void* stream);

/* Atmosphere refresh (reference atm_refresh.py:36-122), uniform batches:
 * mu = ymix . mol_mass per layer; the hydrostatic integration upward from
 * the reference layer pref_indx (zco[pref] = zco_pref, g = gs there) and
 * downward below it, g = gs (Rp / (Rp + zco))^2, Hp = kb T / (mu / Navo g),
 * dz = Hp ln(pico[j] / pico[j+1]); dzi, Hpi the means of adjacent layers;
 * the diffusion-limited escape flux at the top of each esc_idx species,
 * -Dzz_top y_top (1/Hp_top - ms g_top / (Navo kb T_top)), floored at
 * -max_flux. g, dzi, Hpi and those top_flux entries are written into the
 * atmosphere blob (the splice of outer_loop.py:729-730); Tco, ms and Dzz
 * (its last interface row) are read from it. Device arrays: pico
 * [B][nz+1], mol_mass [ni], esc_idx [n_esc], y, ymix [B][nz][ni]; outputs
 * (each nullable) mu, Hp, dz [B][nz], zco [B][nz+1]. */
typedef struct VbRefreshParams {
  int32_t pref_indx, n_esc;
  double zco_pref, gs, Rp, kb, Navo, max_flux;
} VbRefreshParams;
int vb_atm_refresh(int batch, int nz, int ni, const VbRefreshParams* params, const double* pico,
                   const double* mol_mass, const int32_t* esc_idx, const double* y, const double* ymix, double* atm,
                   double* mu, double* Hp, double* dz, double* zco, void* stream);
/* The refresh inside the adaptive loop (outer_loop.py:813-840), after
 * vb_loop_body: for each atmosphere whose attempt was taken (accepted or
 * force-accepted, scalars[b].last_decision != 0) with a pre-increment
 * accept count that is a multiple of update_frq, and that is not done
 * (conv nullable), vb_atm_refresh of the attempt's clipped state (the
 * body's pre_y, pre_ymix); the others are left untouched. */
int vb_loop_refresh(int batch, int nz, int ni, const VbRefreshParams* params, int32_t update_frq,
                    const VbLoopScalars* scalars, const VbConvState* conv, const double* pico,
                    const double* mol_mass, const int32_t* esc_idx, const double* pre_y, const double* pre_ymix,
                    double* atm, double* mu, double* Hp, double* dz, double* zco, void* stream);
/* Condensation inside the adaptive loop (reference outer_loop.py:770-800), after
 * vb_loop_body (with pre_y, pre_ymix, pre_td) and before vb_loop_refresh:
 * for each atmosphere whose attempt was taken with a start time t >=
 * start_conden_time (and that is not done), the condensation rows of k from
 * the attempt's clipped state (conden.py:55-71), then the H2O and NH3
 * cold-trap relaxations with the attempt's dt (conden.py:74-160) applied to
 * that state; for an accepted attempt the hydrostatic rebalance of the body
 * (outer_loop.py:844-917) is redone from the relaxed state: y, y_prev, ymix,
 * atom_loss and atom_loss_prev. The fixed-species switch that the reference
 * couples to the end of the window is not part of it. Device arrays in the
 * table: re_idx, sp_idx, coeff [n_re]; Dg_re, sat_re [B][n_re][nz];
 * h2o_Dg, h2o_sat, nh3_Dg, nh3_sat [B][nz] (nullable when inactive). */
typedef struct VbCondenLoop {
  int32_t n_re, h2o_active, h2o_sp, h2o_l_s, nh3_active, nh3_sp, nh3_l_s, nh3_conden_top;
  double start_conden_time, h2o_m_over_rho_r2, nh3_m_over_rho_r2;
  const int32_t* re_idx;
  const int32_t* sp_idx;
  const double* coeff;
  const double* Dg_re;
  const double* sat_re;
  const double* h2o_Dg;
  const double* h2o_sat;
  const double* nh3_Dg;
  const double* nh3_sat;
} VbCondenLoop;
int vb_loop_condense(int batch, int nz, int ni, int nr, const VbCondenLoop* conden, const VbLoopParams* params,
                     const double* atm, const uint8_t* gas_mask, const double* compo, const double* atom_ini,
                     const VbLoopScalars* scalars, const VbConvState* conv, const double* pre_td, double* pre_y,
                     double* pre_ymix, double* y, double* y_prev, double* ymix, double* atom_loss,
                     double* atom_loss_prev, double* k, void* stream);
/* Condensation rates (reference conden.py:55-71): rate = Dg coeff (y[sp] -
 * sat_n) for each condensation reaction r; k[re_idx[r]] = max(rate, 0),
 * k[re_idx[r] + 1] = max(-rate, 0). Dg, sat_n [B][n_re][nz], coeff [n_re],
 * re_idx, sp_idx [n_re], y [B][nz][ni], k [B][nr+1][nz]. */
int vb_conden_rates(int batch, int nz, int ni, int nr, int n_re, const int32_t* re_idx, const int32_t* sp_idx,
                    const double* coeff, const double* Dg, const double* sat_n, const double* y, double* k,
                    void* stream);
/* Cold-trap relaxation of one condensing species (reference conden.py:74-160):
 * implicit Euler toward saturation, mass moved between species sp and its
 * condensate sp_l_s, then y = ymix * (gas sum of y before the update) for
 * every species. conden_top >= 0 clamps condensation to layers <=
 * conden_top and clips the condensate's ymix at 0 (the NH3 form); -1 is
 * the H2O form. Dg, sat [B][nz], dt [B]; n_0 and the gas mask are the
 * blob's M and gas slots; y, ymix [B][nz][ni] updated in place. */
typedef struct VbRelaxParams {
  int32_t sp, sp_l_s, conden_top, reserved;
  double m_over_rho_r2;
} VbRelaxParams;
int vb_conden_relax(int batch, int nz, int ni, const VbRelaxParams* params, const double* Dg, const double* sat,
                    const double* atm, const double* dt, double* y, double* ymix, void* stream);

/* Profiling: while enabled, every kernel launch of vb_ros2_step is bracketed
 * by CUDA events recorded on the launching stream (launch sites:
 * 0 stage-1 assembly, 1 factor, 2 back sweep 1, 3 stage-2 assembly,
 * 4 forward sweep 2, 5 back sweep 2). vb_profile_read synchronises, writes
 * the summed milliseconds and launch counts of the first n sites, and clears. */
#define VB_PROFILE_SITES 8
int vb_profile(int enable);
int vb_profile_read(double* ms, int64_t* counts, int n);

/* FP64 throughput probe: a register-resident dependent-FMA loop (8 chains per
 * thread) over the whole GPU, writes a checksum to out[0]. Used to measure the
 * FP64 FMA peak that bounds the block factorisation. */
int vb_fp64_probe(double* out, int blocks, int threads, int iters, void* stream);

/* Ros2 step with no caller workspace and no allocation. No counterpart in the
 * reference: it serves callers that cannot cudaMalloc (a host runtime that
 * owns all device memory and hands a foreign call no scratch). Same launch
 * sequence and results as vb_ros2_step for a uniform batch (zoff = NULL),
 * with the workspace in a module-scope device array of
 * VB_STATIC_SCRATCH_BYTES that every device loading the library holds until
 * the process exits. Batches whose vb_ros2_workspace_bytes(batch, nz, ni,
 * NULL) exceeds that maximum are rejected with VB_ERR_ARG. The first call on
 * each device looks the array's device address up (cudaGetSymbolAddress)
 * with that device current; make that first call before any stream capture.
 * All calls on a device share the array and it keeps the last call's
 * contents: calls that overlap on the GPU (streams without an ordering
 * between them) race. Nothing in the array needs to start at zero (every
 * value is written before it is read); status[B] is cleared by each call.
 * The looked-up address is cached per device for the life of the process: a
 * device reset (cudaDeviceReset, or the primary context destroyed and
 * recreated) makes it stale, so this entry point must not be called again in
 * a process after its device was reset. */
#define VB_STATIC_SCRATCH_BYTES ((size_t)64 << 20)
int vb_ros2_step_static(const VbNet* net, int batch, int nz,
                        const double* y, const double* k, const double* dt,
                        const double* atm, int32_t atm_flags, const uint8_t* fix_mask,
                        double* sol, double* delta, int32_t* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VULCAN_B200_H */
