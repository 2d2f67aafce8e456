"""CPU oracle: a NumPy/SciPy FP64 restatement of the reference Ros2 step.

TEST INFRASTRUCTURE ONLY. This module is the checker for the CUDA path: only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import it. The product path never calls it.

It follows, expression by expression, the reference functions:

* ``chem_rhs`` / ``chem_jac_analytical``  -> `chem.py:83-131`, `chem.py:144-214`
* ``compute_diff_grav``                   -> `jax_step.py:67-147`
* ``build_diff_coeffs``                   -> `jax_step.py:150-220`
* ``apply_diffusion``                     -> `jax_step.py:223-246`
* ``ros2_step``                           -> `jax_step.py:249-315`
* ``factor_block_thomas`` / ``solve_block_thomas`` -> `solver.py:33-112`
  (partial-pivot getrf/getrs from SciPy, the same LAPACK algorithm class as
  ``jax.scipy.linalg.lu_factor/lu_solve``; the explicit ``lu_solve(eye)``
  inverse of `solver.py:46` is kept for order-of-operations parity)
* ``block_thomas_dense``                  -> `solver.py:129-178`

The segment sums of `chem.py:113-124,202-207` (``jax.ops.segment_sum``) are
restated with ``numpy.add.at``, which accumulates in increasing flat-index
order. Layers are vectorised (the reference vmaps over them); the arithmetic
per layer is unchanged.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

KB = 1.38064852e-16   # reference phy_const.py:3
NAVO = 6.02214086e23  # reference phy_const.py:4
R_ROS2 = 1.0 + 1.0 / np.sqrt(2.0)


# ----------------------------------------------------------------------------
# chemistry (chem.py)
# ----------------------------------------------------------------------------
def _factors(y, net):
    """y_r**st with the st>0 guard, for every (reaction, slot). [nz, nr+1, T]."""
    nz = y.shape[0]
    yp = np.concatenate([y, np.ones((nz, 1))], axis=1)        # chem.py:92
    y_r = yp[:, net.reactant_idx]                              # chem.py:94
    st = net.reactant_stoich[None]
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        f = np.where(st > 0, y_r ** st, 1.0)                   # chem.py:96
    return y_r, f


def rates(y, M, k, net):
    """rate[z, r] = k[r, z] * prod_slot factor (* M if three-body). chem.py:94-99."""
    _, f = _factors(y, net)
    prod = f[:, :, 0].copy()
    for s in range(1, f.shape[2]):                             # jnp.prod, left to right
        prod = prod * f[:, :, s]
    rate = k.T * prod
    rate = np.where(net.is_three_body[None, :], rate * M[:, None], rate)
    return rate


def chem_rhs(y, M, k, net):
    """dy/dt from chemistry, [nz, ni]. chem.py:83-131."""
    nz, ni = y.shape
    T = net.reactant_idx.shape[1]
    rate = rates(y, M, k, net)                                 # [nz, nr+1]
    rate_rep = np.repeat(rate, T, axis=1)                      # chem.py:105
    r_idx = net.reactant_idx.reshape(-1)
    p_idx = net.product_idx.reshape(-1)
    r_st = net.reactant_stoich.reshape(-1)
    p_st = net.product_stoich.reshape(-1)
    loss = np.zeros((ni + 1, nz), dtype=rate.dtype)            # complex for complex-step derivatives
    prod = np.zeros((ni + 1, nz), dtype=rate.dtype)
    np.add.at(loss, r_idx, (r_st[None, :] * rate_rep).T)       # chem.py:113-118
    np.add.at(prod, p_idx, (p_st[None, :] * rate_rep).T)       # chem.py:119-124
    return (prod[:ni] - loss[:ni]).T


def chem_jac(y, M, k, net):
    """Analytic chemistry Jacobian J[z, i, j] = d(dy_i/dt)/dy_j. chem.py:144-214."""
    nz, ni = y.shape
    T = net.reactant_idx.shape[1]
    y_r, f = _factors(y, net)
    slots = np.arange(T)
    cols = []
    for j in range(T):                                         # chem.py:165-169
        fe = np.where((slots == j)[None, None, :], 1.0, f)
        p = fe[:, :, 0].copy()
        for s in range(1, T):
            p = p * fe[:, :, s]
        cols.append(p)
    leave_out = np.stack(cols, axis=2)                         # [nz, nr+1, T]
    st = net.reactant_stoich[None]
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        pm1 = np.where(st > 0, y_r ** (st - 1.0), 0.0)         # chem.py:173-177
    drate = st * pm1 * leave_out * k.T[:, :, None]             # chem.py:178-180
    drate = np.where(net.is_three_body[None, :, None], drate * M[:, None, None], drate)
    out_idx = np.concatenate([net.reactant_idx, net.product_idx], axis=1)       # [nr+1, 2T]
    out_st = np.concatenate([-net.reactant_stoich, net.product_stoich], axis=1)
    contrib = out_st[None, :, :, None] * drate[:, :, None, :]  # [nz, nr+1, 2T, T]
    row = np.broadcast_to(out_idx[:, :, None], contrib.shape[1:])
    col = np.broadcast_to(net.reactant_idx[:, None, :], contrib.shape[1:])
    keys = (row * (ni + 1) + col).reshape(-1)
    J = np.zeros(((ni + 1) * (ni + 1), nz))
    np.add.at(J, keys, contrib.reshape(nz, -1).T)              # chem.py:202-207
    return J.T.reshape(nz, ni + 1, ni + 1)[:, :ni, :ni]


def chem_rhs_loop(y, M, k, net):
    """Explicit reaction loop (reference `chem.py:217-243`), a second RHS check."""
    nz, ni = y.shape
    dydt = np.zeros_like(y)
    T = net.reactant_idx.shape[1]
    for i in range(1, net.nr + 1):
        rate = np.asarray(k[i], dtype=np.float64).copy()
        for s in range(T):
            sp, st = net.reactant_idx[i, s], net.reactant_stoich[i, s]
            if st == 0:
                continue
            rate = rate * y[:, sp] ** st
        if net.is_three_body[i]:
            rate = rate * M
        for s in range(T):
            sp, st = net.product_idx[i, s], net.product_stoich[i, s]
            if st == 0 or sp >= ni:
                continue
            dydt[:, sp] += st * rate
        for s in range(T):
            sp, st = net.reactant_idx[i, s], net.reactant_stoich[i, s]
            if st == 0 or sp >= ni:
                continue
            dydt[:, sp] -= st * rate
    return dydt


# ----------------------------------------------------------------------------
# diffusion (jax_step.py)
# ----------------------------------------------------------------------------
def compute_diff_grav(atm):
    """y-independent molecular-diffusion pieces. jax_step.py:67-147."""
    dzi, Hpi, Ti, Tco, g, ms, alpha, Dzz = (atm["dzi"], atm["Hpi"], atm["Ti"], atm["Tco"],
                                            atm["g"], atm["ms"], atm["alpha"], atm["Dzz"])
    vm, vs = atm["vm"], atm["vs"]
    nz = Tco.shape[0]
    j = np.arange(1, nz - 1)
    dz_ave = 0.5 * (dzi[j - 1] + dzi[j])
    use_vm = float(bool(atm["use_vm_mol"]))
    use_set = float(bool(atm["use_settling"]))
    C = lambda a: a[:, None]  # noqa: E731
    grav_j = -1.0 / C(Hpi[j]) + ms[None, :] * C(g[j]) / (NAVO * KB * C(Ti[j])) \
        + alpha[None, :] / C(Ti[j]) * (C(Tco[j + 1]) - C(Tco[j])) / C(dzi[j])
    grav_jm = -1.0 / C(Hpi[j - 1]) + ms[None, :] * C(g[j]) / (NAVO * KB * C(Ti[j - 1])) \
        + alpha[None, :] / C(Ti[j - 1]) * (C(Tco[j]) - C(Tco[j - 1])) / C(dzi[j - 1])
    grav_jp_b = -1.0 / C(Hpi[j]) + ms[None, :] * C(g[j + 1]) / (NAVO * KB * C(Ti[j])) \
        + alpha[None, :] / C(Ti[j]) * (C(Tco[j + 1]) - C(Tco[j])) / C(dzi[j])
    grav_jm_c = -1.0 / C(Hpi[j - 1]) + ms[None, :] * C(g[j - 1]) / (NAVO * KB * C(Ti[j - 1])) \
        + alpha[None, :] / C(Ti[j - 1]) * (C(Tco[j]) - C(Tco[j - 1])) / C(dzi[j - 1])
    inv_2dz = 1.0 / (2.0 * C(dz_ave))
    A_grav = inv_2dz * (Dzz[j] * grav_j - Dzz[j - 1] * grav_jm)
    B_grav = inv_2dz * Dzz[j] * grav_jp_b
    C_grav = -inv_2dz * Dzz[j - 1] * grav_jm_c
    bdry0 = (1.0 / dzi[0] * Dzz[0] / 2.0
             * (-1.0 / Hpi[0] + ms * g[0] / (NAVO * KB * Ti[0])
                + alpha / Ti[0] * (Tco[1] - Tco[0]) / dzi[0]))
    bdry_top = (-1.0 / dzi[-1] * Dzz[-1] / 2.0
                * (-1.0 / Hpi[-1] + ms * g[-1] / (NAVO * KB * Ti[-1])
                   + alpha / Ti[-1] * (Tco[-1] - Tco[-2]) / dzi[-1]))
    pos = lambda a: (a > 0) * a  # noqa: E731
    neg = lambda a: (a < 0) * a  # noqa: E731
    A_vm = -(pos(vm[j]) - neg(vm[j - 1])) / C(dz_ave)
    B_vm = -(neg(vm[j])) / C(dz_ave)
    C_vm = (pos(vm[j - 1])) / C(dz_ave)
    b0_vm = -(pos(vm[0])) / dzi[0]
    b0_vm_B = -(neg(vm[0])) / dzi[0]
    bt_vm = (neg(vm[-1])) / dzi[-1]
    bt_vm_C = (pos(vm[-1])) / dzi[-1]
    A_vs = -(pos(vs[j]) - neg(vs[j - 1])) / C(dz_ave)
    B_vs = -(neg(vs[j])) / C(dz_ave)
    C_vs = (pos(vs[j - 1])) / C(dz_ave)
    b0_vs = -(pos(vs[0])) / dzi[0]
    b0_vs_B = -(neg(vs[0])) / dzi[0]
    bt_vs = (neg(vs[-1])) / dzi[-1]
    bt_vs_C = (pos(vs[-1])) / dzi[-1]
    A_base = (1.0 - use_vm) * A_grav + use_vm * A_vm
    B_base = (1.0 - use_vm) * B_grav + use_vm * B_vm
    C_base = (1.0 - use_vm) * C_grav + use_vm * C_vm
    b0_A = (1.0 - use_vm) * bdry0 + use_vm * b0_vm
    b0_B = (1.0 - use_vm) * bdry0 + use_vm * b0_vm_B
    bt_A = (1.0 - use_vm) * bdry_top + use_vm * bt_vm
    bt_C = (1.0 - use_vm) * bdry_top + use_vm * bt_vm_C
    return dict(
        A_grav_int=A_base + use_set * A_vs,
        B_grav_int=B_base + use_set * B_vs,
        C_grav_int=C_base + use_set * C_vs,
        bdry0_grav=np.stack([b0_A + use_set * b0_vs, b0_B + use_set * b0_vs_B]),
        bdry_top_grav=np.stack([bt_A + use_set * bt_vs, bt_C + use_set * bt_vs_C]),
        dz_ave=dz_ave,
    )


def build_diff_coeffs(y, atm, grav):
    """Eddy + molecular coefficients at state y. jax_step.py:150-220."""
    Kzz, Dzz, dzi, vz = atm["Kzz"], atm["Dzz"], atm["dzi"], atm["vz"]
    nz, ni = y.shape
    ysum = np.sum(np.where(np.asarray(atm["gas_indx_mask"], bool)[None, :], y, 0.0), axis=1)
    j = np.arange(1, nz - 1)
    dz_ave = grav["dz_ave"]
    A_e = -1.0 / dz_ave * (
        Kzz[j] / dzi[j] * (ysum[j + 1] + ysum[j]) / 2.0
        + Kzz[j - 1] / dzi[j - 1] * (ysum[j] + ysum[j - 1]) / 2.0) / ysum[j]
    B_e = 1.0 / dz_ave * Kzz[j] / dzi[j] * (ysum[j + 1] + ysum[j]) / 2.0 / ysum[j + 1]
    C_e = 1.0 / dz_ave * Kzz[j - 1] / dzi[j - 1] * (ysum[j] + ysum[j - 1]) / 2.0 / ysum[j - 1]
    A_e = A_e - ((vz[j] > 0) * vz[j] - (vz[j - 1] < 0) * vz[j - 1]) / dz_ave
    B_e = B_e - ((vz[j] < 0) * vz[j]) / dz_ave
    C_e = C_e + ((vz[j - 1] > 0) * vz[j - 1]) / dz_ave
    A0 = -1.0 / dzi[0] * (Kzz[0] / dzi[0]) * (ysum[1] + ysum[0]) / 2.0 / ysum[0]
    A0 = A0 - ((vz[0] > 0) * vz[0]) / dzi[0]
    B0 = 1.0 / dzi[0] * (Kzz[0] / dzi[0]) * (ysum[1] + ysum[0]) / 2.0 / ysum[1]
    B0 = B0 - ((vz[0] < 0) * vz[0]) / dzi[0]
    At = -1.0 / dzi[-1] * (Kzz[-1] / dzi[-1]) * (ysum[-1] + ysum[-2]) / 2.0 / ysum[-1]
    At = At + ((vz[-1] < 0) * vz[-1]) / dzi[-1]
    Ct = 1.0 / dzi[-1] * (Kzz[-1] / dzi[-1]) * (ysum[-1] + ysum[-2]) / 2.0 / ysum[-2]
    Ct = Ct + ((vz[-1] > 0) * vz[-1]) / dzi[-1]
    A_eddy = np.concatenate([[A0], A_e, [At]])
    B_eddy = np.concatenate([[B0], B_e, [0.0]])
    C_eddy = np.concatenate([[0.0], C_e, [Ct]])
    C = lambda a: a[:, None]  # noqa: E731
    Ai = -1.0 / C(dz_ave) * (
        Dzz[j] / C(dzi[j]) * (C(ysum[j + 1]) + C(ysum[j])) / 2.0
        + Dzz[j - 1] / C(dzi[j - 1]) * (C(ysum[j]) + C(ysum[j - 1])) / 2.0) / C(ysum[j])
    Ai = Ai + grav["A_grav_int"]
    Bi = 1.0 / C(dz_ave) * Dzz[j] / C(dzi[j]) * (C(ysum[j + 1]) + C(ysum[j])) / 2.0 / C(ysum[j + 1])
    Bi = Bi + grav["B_grav_int"]
    Ci = 1.0 / C(dz_ave) * Dzz[j - 1] / C(dzi[j - 1]) * (C(ysum[j]) + C(ysum[j - 1])) / 2.0 / C(ysum[j - 1])
    Ci = Ci + grav["C_grav_int"]
    Ai0 = -1.0 / dzi[0] * (Dzz[0] / dzi[0]) * (ysum[1] + ysum[0]) / 2.0 / ysum[0] + grav["bdry0_grav"][0]
    Bi0 = 1.0 / dzi[0] * (Dzz[0] / dzi[0]) * (ysum[1] + ysum[0]) / 2.0 / ysum[1] + grav["bdry0_grav"][1]
    Ait = -1.0 / dzi[-1] * (Dzz[-1] / dzi[-1]) * (ysum[-1] + ysum[-2]) / 2.0 / ysum[-1] + grav["bdry_top_grav"][0]
    Cit = 1.0 / dzi[-1] * (Dzz[-1] / dzi[-1]) * (ysum[-1] + ysum[-2]) / 2.0 / ysum[-2] + grav["bdry_top_grav"][1]
    A_mol = np.concatenate([Ai0[None], Ai, Ait[None]], axis=0)
    B_mol = np.concatenate([Bi0[None], Bi, np.zeros((1, ni))], axis=0)
    C_mol = np.concatenate([np.zeros((1, ni)), Ci, Cit[None]], axis=0)
    return A_eddy, B_eddy, C_eddy, A_mol, B_mol, C_mol, ysum


def apply_diffusion(y, A_eddy, B_eddy, C_eddy, A_mol, B_mol, C_mol, atm):
    """diff[j] = (A+Ai)y[j] + (B+Bi)y[j+1] + (C+Ci)y[j-1] + BC fluxes. jax_step.py:223-246."""
    A = A_eddy[:, None] + A_mol
    B = B_eddy[:, None] + B_mol
    C = C_eddy[:, None] + C_mol
    d0 = A[0] * y[0] + B[0] * y[1]
    dt_ = A[-1] * y[-1] + C[-1] * y[-2]
    di = A[1:-1] * y[1:-1] + B[1:-1] * y[2:] + C[1:-1] * y[:-2]
    diff = np.concatenate([d0[None], di, dt_[None]], axis=0)
    if atm["use_topflux"]:
        diff[-1] = diff[-1] + atm["top_flux"] / atm["dzi"][-1]
    else:
        diff[-1] = diff[-1] + np.zeros_like(atm["top_flux"])
    if atm["use_botflux"]:
        diff[0] = diff[0] + (atm["bot_flux"] - y[0] * atm["bot_vdep"]) / atm["dzi"][0]
    else:
        diff[0] = diff[0] + np.zeros_like(atm["bot_flux"])
    return diff


def diffusion(y, atm, grav=None):
    if grav is None:
        grav = compute_diff_grav(atm)
    co = build_diff_coeffs(y, atm, grav)
    return apply_diffusion(y, *co[:6], atm), co


# ----------------------------------------------------------------------------
# block-tridiagonal Thomas (solver.py)
# ----------------------------------------------------------------------------
def factor_block_thomas(diag, sup_d, sub_d):
    """Factor once; returns (lu[nz], piv[nz], sup_d, sub_d). solver.py:33-64."""
    nz, ni, _ = diag.shape
    eye = np.eye(ni)
    lus = np.empty_like(diag)
    pivs = np.empty((nz, ni), dtype=np.int32)
    lu, piv = sla.lu_factor(diag[0], check_finite=False)
    lus[0], pivs[0] = lu, piv
    for j in range(1, nz):
        inv = sla.lu_solve((lu, piv), eye, check_finite=False)           # solver.py:46
        A_new = diag[j] - (sub_d[j - 1][:, None] * sup_d[j - 1][None, :]) * inv   # :47
        lu, piv = sla.lu_factor(A_new, check_finite=False)              # :48
        lus[j], pivs[j] = lu, piv
    return lus, pivs, sup_d, sub_d


def solve_block_thomas(factors, rhs):
    """Solve with stored factors. solver.py:67-112."""
    lus, pivs, sup_d, sub_d = factors
    nz = rhs.shape[0]
    rmod = np.empty_like(rhs)
    rmod[0] = rhs[0]
    for j in range(1, nz):
        inv_r = sla.lu_solve((lus[j - 1], pivs[j - 1]), rmod[j - 1], check_finite=False)
        rmod[j] = rhs[j] - sub_d[j - 1] * inv_r                          # solver.py:76
    out = np.empty_like(rhs)
    out[-1] = sla.lu_solve((lus[-1], pivs[-1]), rmod[-1], check_finite=False)
    for j in range(nz - 2, -1, -1):
        loc = rmod[j] - sup_d[j] * out[j + 1]                            # solver.py:98
        out[j] = sla.lu_solve((lus[j], pivs[j]), loc, check_finite=False)
    return out


def block_thomas(diag, sup_d, sub_d, rhs):
    """Factor + solve. solver.py:115-126."""
    return solve_block_thomas(factor_block_thomas(diag, sup_d, sub_d), rhs)


def block_thomas_dense(diag, sup, sub, rhs):
    """Generic dense block Thomas (dense off-diagonal blocks). solver.py:129-178."""
    nz = diag.shape[0]
    lu = sla.lu_factor(diag[0], check_finite=False)
    lus = [lu]
    rmod = [rhs[0]]
    for j in range(1, nz):
        invA_B = sla.lu_solve(lus[-1], sup[j - 1], check_finite=False)
        invA_r = sla.lu_solve(lus[-1], rmod[-1], check_finite=False)
        A_new = diag[j] - sub[j - 1] @ invA_B
        rmod.append(rhs[j] - sub[j - 1] @ invA_r)
        lus.append(sla.lu_factor(A_new, check_finite=False))
    out = [None] * nz
    out[-1] = sla.lu_solve(lus[-1], rmod[-1], check_finite=False)
    for j in range(nz - 2, -1, -1):
        out[j] = sla.lu_solve(lus[j], rmod[j] - sup[j] @ out[j + 1], check_finite=False)
    return np.stack(out)


# ----------------------------------------------------------------------------
# the step (jax_step.py:249-315)
# ----------------------------------------------------------------------------
def lhs_blocks(y, k, dt, atm, net, fix_mask=None, grav=None):
    """LHS blocks and stage-1 RHS of the Ros2 step (jax_step.py:257-298).

    Returns (diag[nz,ni,ni], sup_neg[nz-1,ni], sub_neg[nz-1,ni], rhs_y[nz,ni], grav).
    """
    r = 1.0 + 1.0 / np.sqrt(2.0)
    c0 = 1.0 / (r * dt)
    nz, ni = y.shape
    M = atm["M"]
    if grav is None:
        grav = compute_diff_grav(atm)
    A_e, B_e, C_e, A_m, B_m, C_m, _ = build_diff_coeffs(y, atm, grav)
    diff_y = apply_diffusion(y, A_e, B_e, C_e, A_m, B_m, C_m, atm)
    rhs_y = chem_rhs(y, M, k, net) + diff_y
    J = chem_jac(y, M, k, net)
    diag_d = A_e[:, None] + A_m
    sup_d = B_e[:-1, None] + B_m[:-1]
    sub_d = C_e[1:, None] + C_m[1:]
    if atm["use_botflux"]:
        diag_d[0] = diag_d[0] + (-atm["bot_vdep"] / atm["dzi"][0])
    else:
        diag_d[0] = diag_d[0] + np.zeros_like(atm["bot_vdep"])
    di = np.arange(ni)
    diag = c0 * np.eye(ni)[None] - J
    diag[:, di, di] = diag[:, di, di] + (-diag_d)
    sup_neg = -sup_d
    sub_neg = -sub_d
    if fix_mask is not None:
        fm = np.asarray(fix_mask, bool)
        diag = np.where(fm[:, :, None], 0.0, diag)
        dd = diag[:, di, di]
        diag[:, di, di] = np.where(fm, c0, dd)
        rhs_y = np.where(fm, 0.0, rhs_y)
        sup_neg = np.where(fm[:-1], 0.0, sup_neg)
        sub_neg = np.where(fm[1:], 0.0, sub_neg)
    return diag, sup_neg, sub_neg, rhs_y, grav


def ros2_step(y, k, dt, atm, net, fix_mask=None, return_parts=False):
    """One 2nd-order Rosenbrock step -> (sol, delta_arr). jax_step.py:249-315."""
    r = 1.0 + 1.0 / np.sqrt(2.0)
    M = atm["M"]
    diag, sup_neg, sub_neg, rhs_y, grav = lhs_blocks(y, k, dt, atm, net, fix_mask)
    factors = factor_block_thomas(diag, sup_neg, sub_neg)
    k1 = solve_block_thomas(factors, rhs_y)
    yk2 = y + k1 / r
    A_e, B_e, C_e, A_m, B_m, C_m, _ = build_diff_coeffs(yk2, atm, grav)
    diff2 = apply_diffusion(yk2, A_e, B_e, C_e, A_m, B_m, C_m, atm)
    rhs_yk2 = chem_rhs(yk2, M, k, net) + diff2
    if fix_mask is not None:
        rhs_yk2 = np.where(np.asarray(fix_mask, bool), 0.0, rhs_yk2)
    rhs2 = rhs_yk2 - (2.0 / (r * dt)) * k1
    k2 = solve_block_thomas(factors, rhs2)
    sol = y + (3.0 / (2.0 * r)) * k1 + (1.0 / (2.0 * r)) * k2
    delta = np.abs(sol - yk2)
    if return_parts:
        return sol, delta, dict(k1=k1, k2=k2, yk2=yk2, rhs_y=rhs_y, rhs2=rhs2, diag=diag,
                                sup_neg=sup_neg, sub_neg=sub_neg)
    return sol, delta


def integrate_fixed_dt(y0, k, dt, n_steps, atm, net):
    """N fixed-dt steps; per-step max relative delta. integrate.py:20-36."""
    y = y0
    deltas = []
    for _ in range(n_steps):
        sol, d = ros2_step(y, k, dt, atm, net)
        deltas.append(np.max(d / np.maximum(np.abs(sol), 1e-30)))
        y = sol
    return y, np.array(deltas)


def chem_rhs_abs(y, M, k, net):
    """Sum of |terms| of each species' RHS gather (the scale of its rounding
    error bound): sum over slots of |st * rate| for losses and productions."""
    return np.abs(chem_rhs_terms(y, M, k, net))


def chem_rhs_terms(y, M, k, net):
    nz, ni = y.shape
    T = net.reactant_idx.shape[1]
    rate = np.abs(rates(y, M, k, net))
    rate_rep = np.repeat(rate, T, axis=1)
    acc = np.zeros((ni + 1, nz))
    np.add.at(acc, net.reactant_idx.reshape(-1), (np.abs(net.reactant_stoich.reshape(-1))[None, :] * rate_rep).T)
    np.add.at(acc, net.product_idx.reshape(-1), (np.abs(net.product_stoich.reshape(-1))[None, :] * rate_rep).T)
    return acc[:ni].T


def chem_jac_abs(y, M, k, net):
    """Sum of |contributions| of each Jacobian entry (its rounding-error scale)."""
    nz, ni = y.shape
    T = net.reactant_idx.shape[1]
    y_r, f = _factors(np.abs(y), net)
    slots = np.arange(T)
    cols = []
    for j in range(T):
        fe = np.where((slots == j)[None, None, :], 1.0, f)
        p = fe[:, :, 0].copy()
        for s in range(1, T):
            p = p * fe[:, :, s]
        cols.append(p)
    leave_out = np.stack(cols, axis=2)
    st = net.reactant_stoich[None]
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        pm1 = np.where(st > 0, y_r ** (st - 1.0), 0.0)
    drate = np.abs(st * pm1 * leave_out * np.abs(k).T[:, :, None])
    drate = np.where(net.is_three_body[None, :, None], drate * np.abs(M)[:, None, None], drate)
    out_idx = np.concatenate([net.reactant_idx, net.product_idx], axis=1)
    out_st = np.abs(np.concatenate([net.reactant_stoich, net.product_stoich], axis=1))
    contrib = out_st[None, :, :, None] * drate[:, :, None, :]
    row = np.broadcast_to(out_idx[:, :, None], contrib.shape[1:])
    col = np.broadcast_to(net.reactant_idx[:, None, :], contrib.shape[1:])
    keys = (row * (ni + 1) + col).reshape(-1)
    J = np.zeros(((ni + 1) * (ni + 1), nz))
    np.add.at(J, keys, contrib.reshape(nz, -1).T)
    return J.T.reshape(nz, ni + 1, ni + 1)[:, :ni, :ni]


# ----------------------------------------------------------------------------
# checks of a step computed elsewhere (by its two block solves)
# ----------------------------------------------------------------------------
def stage_rhs(y, k, atm, net, fix_mask=None, grav=None):
    """f(y) = chem_rhs + diffusion with boundary fluxes, the right-hand side
    of either Ros2 stage before the k1 term (jax_step.py:275-282, :304-309)."""
    if grav is None:
        grav = compute_diff_grav(atm)
    A_e, B_e, C_e, A_m, B_m, C_m, _ = build_diff_coeffs(y, atm, grav)
    f = chem_rhs(y, atm["M"], k, net) + apply_diffusion(y, A_e, B_e, C_e, A_m, B_m, C_m, atm)
    if fix_mask is not None:
        f = np.where(np.asarray(fix_mask, bool), 0.0, f)
    return f


def block_apply(diag, sup_n, sub_n, x):
    """M x for the block-tridiagonal system of solver.py:33-112 (dense
    diagonal blocks, diagonal off-diagonal blocks as the solver receives them)."""
    out = np.einsum("zij,zj->zi", diag, x)
    out[:-1] += sup_n * x[1:]
    out[1:] += sub_n * x[:-1]
    return out


def backward_error(diag, sup_n, sub_n, x, rhs):
    """Normwise backward error ||M x - rhs||_inf / (||M||_inf ||x||_inf + ||rhs||_inf)
    of a computed solution x of the block system."""
    res = block_apply(diag, sup_n, sub_n, x) - rhs
    normM = np.abs(diag).sum(axis=2)
    normM[:-1] += np.abs(sup_n)
    normM[1:] += np.abs(sub_n)
    den = normM.max() * np.abs(x).max() + np.abs(rhs).max()
    return float(np.abs(res).max() / den) if den > 0 else float(np.abs(res).max())


def stage_backward_errors(y, k, dt, atm, net, k1, k2, fix_mask=None):
    """Backward errors of the two block solves of a Ros2 step whose stage
    vectors k1, k2 were computed elsewhere: LHS k1 = f(y) and
    LHS k2 = f(y + k1/r) - 2/(r dt) k1 (jax_step.py:300-311), with the LHS and
    right-hand sides built here in FP64. Returns (bwd1, bwd2)."""
    diag, sup_n, sub_n, rhs1, grav = lhs_blocks(y, k, dt, atm, net, fix_mask)
    yk2 = y + k1 / R_ROS2
    rhs2 = stage_rhs(yk2, k, atm, net, fix_mask, grav) - (2.0 / (R_ROS2 * dt)) * k1
    return (backward_error(diag, sup_n, sub_n, k1, rhs1), backward_error(diag, sup_n, sub_n, k2, rhs2))


def schur_block_conditions(diag, sup_n, sub_n):
    """inf-norm condition number of every Schur-updated diagonal block A'_j of
    the factor recursion (solver.py:44-48)."""
    nz, ni, _ = diag.shape
    eye = np.eye(ni)
    conds = np.empty(nz)
    A = diag[0]
    for j in range(nz):
        if j > 0:
            A = diag[j] - (sub_n[j - 1][:, None] * sup_n[j - 1][None, :]) * inv
        lu = sla.lu_factor(A, check_finite=False)
        inv = sla.lu_solve(lu, eye, check_finite=False)
        conds[j] = np.abs(A).sum(axis=1).max() * np.abs(inv).sum(axis=1).max()
    return conds
