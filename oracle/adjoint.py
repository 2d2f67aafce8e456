"""CPU oracle for the implicit steady-state adjoint (reference `steady_state_grad.py`).

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` only.

* ``residual``              -> `steady_state_residual_inputs` (`:116-130`):
  f(y) = chem_rhs(y) + diffusion(y)
* ``jacobian_blocks``       -> `_build_jacobian_blocks` (`:153-175`)
* ``validate``              -> `validate_steady_state_solution` (`:178-196`)
* ``ss_bwd``                -> `_ssi_bwd` (`:214-230`): lambda from the
  transposed block-Thomas solve (reference order: factor ``diag^T`` with
  sup/sub exchanged), then ``-vjp(f)(lambda)`` over the differentiable
  inputs. The VJP is taken with torch autograd (float64) through a torch
  restatement of the same residual expressions (jax_step.py:67-246,
  chem.py:83-131); JAX's ``vjp`` is not available here.
"""
from __future__ import annotations

import numpy as np
import torch

from . import ros2

LEAVES = ["k_arr", "Kzz", "Dzz", "dzi", "vz", "Hpi", "Ti", "Tco", "g", "ms", "alpha", "M", "vm", "vs",
          "top_flux", "bot_flux", "bot_vdep"]


def residual(y, k, atm, net):
    diff, _ = ros2.diffusion(y, atm)
    return ros2.chem_rhs(y, atm["M"], k, net) + diff


def jacobian_blocks(y, k, atm, net):
    """J_y = chem_J + diag(A_eddy + A_mol) (+ deposition), sup = B[:-1], sub = C[1:]."""
    grav = ros2.compute_diff_grav(atm)
    A_e, B_e, C_e, A_m, B_m, C_m, _ = ros2.build_diff_coeffs(y, atm, grav)
    J = ros2.chem_jac(y, atm["M"], k, net)
    diag_d = A_e[:, None] + A_m
    sup = B_e[:-1, None] + B_m[:-1]
    sub = C_e[1:, None] + C_m[1:]
    ni = y.shape[1]
    di = np.arange(ni)
    diag = J.copy()
    diag[:, di, di] = diag[:, di, di] + diag_d
    if atm["use_botflux"]:
        diag[0, di, di] = diag[0, di, di] + (-atm["bot_vdep"] / atm["dzi"][0])
    return diag, sup, sub


def validate(y, k, atm, net, rtol=1e-6, atol=0.0):
    r = residual(y, k, atm, net)
    ri = float(np.max(np.abs(r)))
    tol = max(atol, rtol * max(float(np.max(np.abs(y))), 1.0))
    if ri > tol:
        raise ValueError(f"residual {ri:.3e} exceeds {tol:.3e}")
    return ri


# ---------------------------------------------------------------- torch residual
def _t(x):
    return torch.as_tensor(np.asarray(x, dtype=np.float64))


def residual_torch(y, P, net, flags):
    """f(y, P) with P a dict of float64 torch leaves (names as LEAVES)."""
    Kzz, Dzz, dzi, vz, Hpi, Ti, Tco, g = P["Kzz"], P["Dzz"], P["dzi"], P["vz"], P["Hpi"], P["Ti"], P["Tco"], P["g"]
    ms, alpha, M, vm, vs = P["ms"], P["alpha"], P["M"], P["vm"], P["vs"]
    nz, ni = y.shape
    KB, NAVO = ros2.KB, ros2.NAVO
    use_vm = 1.0 if flags["use_vm_mol"] else 0.0
    use_set = 1.0 if flags["use_settling"] else 0.0
    j = torch.arange(1, nz - 1)
    dz_ave = 0.5 * (dzi[j - 1] + dzi[j])
    C = lambda a: a[:, None]  # noqa: E731
    pos = lambda a: (a > 0).double() * a  # noqa: E731
    neg = lambda a: (a < 0).double() * a  # noqa: E731
    gj = -1.0 / C(Hpi[j]) + ms[None] * C(g[j]) / (NAVO * KB * C(Ti[j])) + alpha[None] / C(Ti[j]) * (C(Tco[j + 1]) - C(Tco[j])) / C(dzi[j])
    gjm = -1.0 / C(Hpi[j - 1]) + ms[None] * C(g[j]) / (NAVO * KB * C(Ti[j - 1])) + alpha[None] / C(Ti[j - 1]) * (C(Tco[j]) - C(Tco[j - 1])) / C(dzi[j - 1])
    gjpb = -1.0 / C(Hpi[j]) + ms[None] * C(g[j + 1]) / (NAVO * KB * C(Ti[j])) + alpha[None] / C(Ti[j]) * (C(Tco[j + 1]) - C(Tco[j])) / C(dzi[j])
    gjmc = -1.0 / C(Hpi[j - 1]) + ms[None] * C(g[j - 1]) / (NAVO * KB * C(Ti[j - 1])) + alpha[None] / C(Ti[j - 1]) * (C(Tco[j]) - C(Tco[j - 1])) / C(dzi[j - 1])
    inv2 = 1.0 / (2.0 * C(dz_ave))
    Ag = inv2 * (Dzz[j] * gj - Dzz[j - 1] * gjm)
    Bg = inv2 * Dzz[j] * gjpb
    Cg = -inv2 * Dzz[j - 1] * gjmc
    b0 = 1.0 / dzi[0] * Dzz[0] / 2.0 * (-1.0 / Hpi[0] + ms * g[0] / (NAVO * KB * Ti[0]) + alpha / Ti[0] * (Tco[1] - Tco[0]) / dzi[0])
    bt = -1.0 / dzi[-1] * Dzz[-1] / 2.0 * (-1.0 / Hpi[-1] + ms * g[-1] / (NAVO * KB * Ti[-1]) + alpha / Ti[-1] * (Tco[-1] - Tco[-2]) / dzi[-1])
    Avm = -(pos(vm[j]) - neg(vm[j - 1])) / C(dz_ave)
    Bvm = -neg(vm[j]) / C(dz_ave)
    Cvm = pos(vm[j - 1]) / C(dz_ave)
    Avs = -(pos(vs[j]) - neg(vs[j - 1])) / C(dz_ave)
    Bvs = -neg(vs[j]) / C(dz_ave)
    Cvs = pos(vs[j - 1]) / C(dz_ave)
    Ax = (1 - use_vm) * Ag + use_vm * Avm + use_set * Avs
    Bx = (1 - use_vm) * Bg + use_vm * Bvm + use_set * Bvs
    Cx = (1 - use_vm) * Cg + use_vm * Cvm + use_set * Cvs
    b0A = (1 - use_vm) * b0 + use_vm * (-pos(vm[0]) / dzi[0]) + use_set * (-pos(vs[0]) / dzi[0])
    b0B = (1 - use_vm) * b0 + use_vm * (-neg(vm[0]) / dzi[0]) + use_set * (-neg(vs[0]) / dzi[0])
    btA = (1 - use_vm) * bt + use_vm * (neg(vm[-1]) / dzi[-1]) + use_set * (neg(vs[-1]) / dzi[-1])
    btC = (1 - use_vm) * bt + use_vm * (pos(vm[-1]) / dzi[-1]) + use_set * (pos(vs[-1]) / dzi[-1])
    gas = torch.as_tensor(np.asarray(flags["gas_indx_mask"], bool))
    ys = torch.where(gas[None], y, torch.zeros_like(y)).sum(1)
    Ae = -1.0 / dz_ave * (Kzz[j] / dzi[j] * (ys[j + 1] + ys[j]) / 2.0 + Kzz[j - 1] / dzi[j - 1] * (ys[j] + ys[j - 1]) / 2.0) / ys[j]
    Be = 1.0 / dz_ave * Kzz[j] / dzi[j] * (ys[j + 1] + ys[j]) / 2.0 / ys[j + 1]
    Ce = 1.0 / dz_ave * Kzz[j - 1] / dzi[j - 1] * (ys[j] + ys[j - 1]) / 2.0 / ys[j - 1]
    Ae = Ae - (pos(vz[j]) - neg(vz[j - 1])) / dz_ave
    Be = Be - neg(vz[j]) / dz_ave
    Ce = Ce + pos(vz[j - 1]) / dz_ave
    A0 = -1.0 / dzi[0] * (Kzz[0] / dzi[0]) * (ys[1] + ys[0]) / 2.0 / ys[0] - pos(vz[0]) / dzi[0]
    B0 = 1.0 / dzi[0] * (Kzz[0] / dzi[0]) * (ys[1] + ys[0]) / 2.0 / ys[1] - neg(vz[0]) / dzi[0]
    At = -1.0 / dzi[-1] * (Kzz[-1] / dzi[-1]) * (ys[-1] + ys[-2]) / 2.0 / ys[-1] + neg(vz[-1]) / dzi[-1]
    Ct = 1.0 / dzi[-1] * (Kzz[-1] / dzi[-1]) * (ys[-1] + ys[-2]) / 2.0 / ys[-2] + pos(vz[-1]) / dzi[-1]
    Ai = -1.0 / C(dz_ave) * (Dzz[j] / C(dzi[j]) * (C(ys[j + 1]) + C(ys[j])) / 2.0 + Dzz[j - 1] / C(dzi[j - 1]) * (C(ys[j]) + C(ys[j - 1])) / 2.0) / C(ys[j]) + Ax
    Bi = 1.0 / C(dz_ave) * Dzz[j] / C(dzi[j]) * (C(ys[j + 1]) + C(ys[j])) / 2.0 / C(ys[j + 1]) + Bx
    Ci = 1.0 / C(dz_ave) * Dzz[j - 1] / C(dzi[j - 1]) * (C(ys[j]) + C(ys[j - 1])) / 2.0 / C(ys[j - 1]) + Cx
    Ai0 = -1.0 / dzi[0] * (Dzz[0] / dzi[0]) * (ys[1] + ys[0]) / 2.0 / ys[0] + b0A
    Bi0 = 1.0 / dzi[0] * (Dzz[0] / dzi[0]) * (ys[1] + ys[0]) / 2.0 / ys[1] + b0B
    Ait = -1.0 / dzi[-1] * (Dzz[-1] / dzi[-1]) * (ys[-1] + ys[-2]) / 2.0 / ys[-1] + btA
    Cit = 1.0 / dzi[-1] * (Dzz[-1] / dzi[-1]) * (ys[-1] + ys[-2]) / 2.0 / ys[-2] + btC
    zero = torch.zeros(1, dtype=torch.float64)
    A = torch.cat([A0[None], Ae, At[None]])[:, None] + torch.cat([Ai0[None], Ai, Ait[None]])
    B = torch.cat([B0[None], Be, zero])[:, None] + torch.cat([Bi0[None], Bi, torch.zeros(1, ni, dtype=torch.float64)])
    Cc = torch.cat([zero, Ce, Ct[None]])[:, None] + torch.cat([torch.zeros(1, ni, dtype=torch.float64), Ci, Cit[None]])
    d0 = A[0] * y[0] + B[0] * y[1]
    dtop = A[-1] * y[-1] + Cc[-1] * y[-2]
    dint = A[1:-1] * y[1:-1] + B[1:-1] * y[2:] + Cc[1:-1] * y[:-2]
    if flags["use_topflux"]:
        dtop = dtop + P["top_flux"] / dzi[-1]
    if flags["use_botflux"]:
        d0 = d0 + (P["bot_flux"] - y[0] * P["bot_vdep"]) / dzi[0]
    diff = torch.cat([d0[None], dint, dtop[None]])
    # chemistry
    T = net.reactant_idx.shape[1]
    yp = torch.cat([y, torch.ones(nz, 1, dtype=torch.float64)], 1)
    ridx = torch.as_tensor(net.reactant_idx)
    st = torch.as_tensor(net.reactant_stoich)
    yr = yp[:, ridx]
    f = torch.where(st[None] > 0, yr ** st[None], torch.ones_like(yr))
    prod = f[:, :, 0]
    for s in range(1, T):
        prod = prod * f[:, :, s]
    rate = P["k_arr"].T * prod
    three = torch.as_tensor(net.is_three_body)
    rate = torch.where(three[None], rate * M[:, None], rate)
    out = torch.zeros(nz, ni + 1, dtype=torch.float64)
    pidx = torch.as_tensor(net.product_idx)
    pst = torch.as_tensor(net.product_stoich)
    for s in range(T):
        out = out.index_add(1, pidx[:, s], pst[None, :, s] * rate)
        out = out.index_add(1, ridx[:, s], -st[None, :, s] * rate)
    return out[:, :ni] + diff


def ss_bwd(y_star, k, atm, net, v):
    """(lambda, cotangents dict) of the implicit adjoint (steady_state_grad.py:214-230)."""
    diag, sup, sub = jacobian_blocks(y_star, k, atm, net)
    lam = ros2.block_thomas(np.transpose(diag, (0, 2, 1)), sub, sup, v)
    return lam, vjp_from_lambda(y_star, k, atm, net, lam)


def vjp_from_lambda(y_star, k, atm, net, lam):
    """-lambda . df/dtheta for every differentiable leaf (steady_state_grad.py:221-229)."""
    P = {name: _t(atm[name] if name != "k_arr" else k).requires_grad_(True) for name in LEAVES}
    flags = {f: atm[f] for f in ("use_vm_mol", "use_settling", "use_topflux", "use_botflux", "gas_indx_mask")}
    f = residual_torch(_t(y_star), P, net, flags)
    grads = torch.autograd.grad(f, [P[n] for n in LEAVES], grad_outputs=_t(lam), allow_unused=True)
    cot = {}
    for n, gr in zip(LEAVES, grads):
        cot[n] = -(gr.numpy() if gr is not None else np.zeros_like(np.asarray(atm[n] if n != "k_arr" else k)))
    return cot


def newton_steady_state(y0, k, atm, net, tol=1e-9, max_iter=100):
    """Newton on f(y) = 0 with the block solver (reference tests/test_steady_state_grad.py:135-154)."""
    y = y0.copy()
    for it in range(max_iter):
        r = residual(y, k, atm, net)
        if np.max(np.abs(r)) < tol:
            return y, it
        diag, sup, sub = jacobian_blocks(y, k, atm, net)
        y = y + ros2.block_thomas(diag, sup, sub, -r)
    raise RuntimeError("Newton did not converge")
