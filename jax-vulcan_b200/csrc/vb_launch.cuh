// Host-side launchers shared by the C-ABI translation unit and the kernel units.
#pragma once
#include <cuda_runtime.h>

#include "vb_common.cuh"

namespace vb {

enum SweepMode { SWEEP_FWD = 0, SWEEP_BACK = 1, SWEEP_BACK_FINAL = 2 };

struct SweepArgs {
  int mode;              // SweepMode
  int transposed;        // solve with A^T (adjoint)
  double* user;          // uniform [B][nz][ni] vector (standalone solves), or nullptr (workspace)
  const double* y;       // SWEEP_BACK_FINAL: state y
  double* sol;           // SWEEP_BACK_FINAL outputs
  double* delta;
  int32_t* status;
};

// adj_v != nullptr: assemble the steady-state Jacobian blocks J_y and copy the
// cotangent adj_v [B][nz][ni] into the right-hand side instead of the Ros2 LHS.
cudaError_t launch_stage1(const NetDev&, const Batch&, const double* y, const double* k, const double* dt,
                          const double* atm, int flags, const uint8_t* fix_mask, double* ws, cudaStream_t,
                          const double* adj_v = nullptr);
// resid != nullptr: write the residual f(y) = chem + diffusion to resid [B][nz][ni]
// instead of the stage-2 right-hand side.
cudaError_t launch_stage2(const NetDev&, const Batch&, const double* y, const double* k, const double* dt,
                          const double* atm, int flags, const uint8_t* fix_mask, double* ws, cudaStream_t,
                          double* resid = nullptr);
// Cotangents from lambda held in the workspace's k1 rows (see vb_adjoint).
cudaError_t launch_vjp_atm(const Batch& B, const double* y, const double* atm, int flags, const double* lam,
                           double* g_atm, cudaStream_t st);
cudaError_t launch_vjp(const NetDev&, const Batch&, const double* y, const double* k, const double* atm, int flags,
                       double* ws, double* g_k, double* g_M, double* g_Kzz, double* g_top, double* g_bot,
                       double* g_vdep, cudaStream_t);
// Stage rows of the workspace: k1 (or the adjoint's lambda) and, with k2 set,
// the Ros2 step's k2, into [layers][ni] arrays (either may be nullptr).
cudaError_t launch_gather_stages(const Batch&, const double* ws, double* k1, double* k2, cudaStream_t);
// Poll limit of the bounded waits of the factor and sweep kernels (a wait that
// runs out sets VB_STATUS_WATCHDOG); polls < 0 restores the default.
void set_wait_limit(long long polls);
void set_pipe_wait_limit(long long polls);
long long wait_limit();
// FP64 factor kernel: 0 = blocked Gauss-Jordan with FP64 tensor-core trailing
// updates, 1 = scalar Gauss-Jordan.
void set_factor_variant(int v);
cudaError_t launch_chem(const NetDev&, int batch, int nz, const double* y, const double* M, const double* k,
                        double* dydt, double* jac, cudaStream_t);
cudaError_t launch_diffusion(int batch, int nz, int ni, const double* y, const double* atm, int flags,
                             double* diff, double* diag_d, double* sup_d, double* sub_d, cudaStream_t);
// Inverts every layer's Schur-updated block. for_transposed_solves: the
// inverses will be applied transposed (the adjoint's sweeps), so the
// elimination bounds |X A' - I| instead of |A' X - I|.
cudaError_t launch_factor(const Batch&, double* ws, int32_t* status, int with_rhs, cudaStream_t,
                          bool for_transposed_solves = false);
cudaError_t launch_sweep(const Batch&, double* ws, const SweepArgs&, cudaStream_t);
cudaError_t launch_pack_blocks(const Batch&, const double* diag, const double* sup_d, const double* sub_d,
                               double* ws, cudaStream_t);

// due (nullable): per-atmosphere mask; achg (nullable): &conv[0].aflux_change
cudaError_t launch_photo_tau(int batch, int nz, int ni, const VbPhoto& P, const double* y, const double* dz,
                             double* tau, const int32_t* due, double* achg, cudaStream_t);
cudaError_t launch_photo_flux(int batch, int nz, int ni, const VbPhoto& P, const double* tau, const double* ymix,
                              const double* du_prev, double* aflux, double* sflux, double* dd, double* du,
                              const int32_t* due, double flux_atol, double* achg, cudaStream_t);
cudaError_t launch_photo_j(int batch, int nz, int nr, const VbPhoto& P, const double* aflux, double* J_br,
                           double* J_br_T, double* k, const int32_t* due, cudaStream_t);
cudaError_t launch_rates(int batch, int nz, const VbRateTables& t, const double* T, const double* M, int flags,
                         double* k, double* dkdT, cudaStream_t st);
cudaError_t launch_atm_refresh(int batch, int nz, int ni, const VbRefreshParams& p, const double* pico,
                               const double* mol_mass, const int32_t* esc, const double* y, const double* ymix,
                               double* atm, double* mu, double* Hp, double* dz, double* zco,
                               const VbLoopScalars* loop_st, int update_frq, const VbConvState* conv,
                               cudaStream_t st);
cudaError_t launch_conden_rates(int batch, int nz, int ni, int nr, int n_re, const int32_t* re_idx,
                                const int32_t* sp_idx, const double* coeff, const double* Dg, const double* sat,
                                const double* y, double* k, cudaStream_t st);
cudaError_t launch_conden_relax(int batch, int nz, int ni, const VbRelaxParams& p, const double* Dg,
                                const double* sat, const double* atm, const double* dt, double* y, double* ymix,
                                cudaStream_t st);
cudaError_t launch_fp64_probe(double* out, int blocks, int threads, int iters, cudaStream_t);
template <typename R>
cudaError_t launch_refine(const Batch& B, double* ws, const R* inv, const void* mxr, const double* rhs, double* x,
                          int32_t* state, int32_t* passes, double tol, int first, const int32_t* only,
                          cudaStream_t st);
// Mixed-precision Ros2 step (vb_mixed.cu): one solve pass (first: x = M~^{-1} b;
// else one FP64-residual refinement pass) over rmod -> k1 (xsel 0) / aux (1).
cudaError_t launch_mx_pass(const Batch& B, double* ws, void* mxr, int xsel, bool first, int32_t* mode,
                           const int32_t* only, int32_t* passes, double tol, int32_t* status, cudaStream_t st);
// op 0: modes after the FP32 factor; op 1: stalled refinements to FP64 (todo)
cudaError_t launch_mx_mode(int batch, int op, int32_t* mode, int32_t* todo, int32_t* status32, int32_t* status,
                           cudaStream_t st);
cudaError_t launch_mx_finish(const Batch& B, const double* ws, const double* y, double* sol, double* delta,
                             int32_t* status, cudaStream_t st);
// FP32 factor of the mixed step: row-equilibrated blocks, blocked Gauss-Jordan
// with 3xTF32 tensor-core trailing updates; inverses and row scales into the
// mixed region, the FP64 blocks stay in the workspace.
cudaError_t launch_factor32(const Batch& B, double* ws, void* mxr, int32_t* status32, cudaStream_t st);
// FP64 factor of the atmospheres with only[b] != 0, in place over their blocks.
cudaError_t launch_factor_only(const Batch& B, double* ws, const int32_t* only, int32_t* status, cudaStream_t st);
cudaError_t launch_refine_finalize(int batch, const int32_t* state, int32_t* fallback, int32_t* status,
                                   cudaStream_t st);
template <typename R>
cudaError_t launch_factor_into(const Batch& B, double* ws, R* out, const int32_t* only, int32_t* status,
                               cudaStream_t st);
cudaError_t launch_loop_body(const Batch& B, const VbLoopParams& p, const uint8_t* gas, const double* compo,
                             const double* atom_ini, const double* atm, const uint8_t* fix_mask,
                             const double* fix_y, const double* sol, const double* delta, double* y,
                             double* y_prev, double* ymix, double* atom_loss, double* atom_loss_prev,
                             double* dt, VbLoopScalars* st, const VbConvState* conv, double* pre_y,
                             double* pre_ymix, double* pre_td, cudaStream_t stream);
cudaError_t launch_loop_condense(int batch, int nz, int ni, int nr, const VbCondenLoop& c, const VbLoopParams& p,
                                 const double* atm, const uint8_t* gas, const double* compo, const double* atom_ini,
                                 const VbLoopScalars* st, const VbConvState* conv, const double* pre_td,
                                 double* pre_y, double* pre_ymix, double* y, double* y_prev, double* ymix,
                                 double* atom_loss, double* atom_loss_prev, double* k, cudaStream_t stream);
cudaError_t launch_loop_conv(const Batch& B, const VbConvParams& p, const double* atm, const double* slope_min,
                             const uint8_t* ignore, const double* y, const double* ymix, const VbLoopScalars* st,
                             double* ring_y, double* ring_t, VbConvState* conv, int32_t* photo_due,
                             cudaStream_t stream);

}  // namespace vb
