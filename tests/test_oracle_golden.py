"""The CPU oracle against fixtures made by running the reference's own code.

The fixtures (``tests/golden/*.npz``) hold the outputs of the unmodified
reference `jax_step.jax_ros2_step`, `chem.chem_rhs` / `chem_jac_analytical`,
`solver.*`, `integrate.jax_integrate_fixed_dt`, `photo.*` and the
`outer_loop.py` caller-contract functions (see ``tests/golden/make_golden.py``).
The oracle restates the same arithmetic, so agreement is expected to the last
bit; the assertions allow 1e-13 relative for platform LAPACK differences.
"""
import numpy as np
import pytest

from conftest import BODY_FIELDS, STEP_CASES, body_kwargs, golden, golden_body, golden_step, load_pkg
from oracle import contract as oc
from oracle import photo as op
from oracle import ros2 as orc

TABLES = ["reactant_idx", "product_idx", "reactant_stoich", "product_stoich", "is_three_body"]


def close(a, b, rtol=1e-13, floor=1e-300):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    same_nonfinite = (~np.isfinite(a)) & (~np.isfinite(b))
    err = np.where(same_nonfinite, 0.0, np.abs(a - b) / np.maximum(np.abs(b), floor))
    assert np.nanmax(err, initial=0.0) <= rtol, np.nanmax(err)


@pytest.mark.parametrize("name", STEP_CASES + ["stiff"])
def test_parser_matches_reference_parser(name):
    net, _, _, _, _, _, g = golden_step(name)
    assert net.ni == int(g["ni"]) and net.nr == int(g["nr"])
    for t in TABLES:
        np.testing.assert_array_equal(getattr(net, t), g["tab_" + t])


@pytest.mark.parametrize("name", STEP_CASES + ["stiff"])
def test_chem_rhs_and_jacobian(name):
    net, atm, y, k, dt, fm, g = golden_step(name)
    close(orc.chem_rhs(y, atm["M"], k, net), g["rhs"], rtol=0.0)
    close(orc.chem_jac(y, atm["M"], k, net), g["jac"], rtol=0.0)


@pytest.mark.parametrize("name", STEP_CASES)
def test_ros2_step(name):
    net, atm, y, k, dt, fm, g = golden_step(name)
    sol, delta = orc.ros2_step(y, k, dt, atm, net, fix_mask=fm)
    close(sol, g["sol"])
    close(delta, g["delta"])


def test_integrate_fixed_dt():
    net, atm, y, k, dt, fm, g = golden_step("plain")
    yN, deltas = orc.integrate_fixed_dt(y, k, dt, int(g["int_n"]), atm, net)
    close(yN, g["int_y"])
    close(deltas, g["int_deltas"])


def test_block_thomas_known_systems():
    g = golden("thomas.npz")
    x = orc.block_thomas_dense(g["dense_small_diag"], g["dense_small_sup"], g["dense_small_sub"],
                               g["dense_small_rhs"])
    close(x, g["dense_small_x"])
    x = orc.block_thomas(g["diag_small_diag"], g["diag_small_sup"], g["diag_small_sub"], g["diag_small_rhs"])
    close(x, g["diag_small_x"])
    # regenerate the (nz=120, ni=93) system of the reference test from its seed
    rng = np.random.default_rng(7)
    nz, ni = 8, 5
    rng.standard_normal((nz, ni, ni)); rng.standard_normal((nz - 1, ni))
    rng.standard_normal((nz - 1, ni)); rng.standard_normal((nz, ni))
    d2 = rng.standard_normal((120, 93, 93)) + 1e10 * np.eye(93)
    su2 = rng.standard_normal((119, 93)) * 1e-3
    sb2 = rng.standard_normal((119, 93)) * 1e-3
    r2 = rng.standard_normal((120, 93))
    np.testing.assert_allclose([d2.sum(), su2.sum(), sb2.sum(), r2.sum()], g["diag_big_checksum"], rtol=1e-12)
    close(orc.block_thomas(d2, su2, sb2, r2), g["diag_big_x"], rtol=1e-12)


def test_block_thomas_vs_dense_solve():
    """Reference tests/test_block_thomas_diag.py:129-192: diag-offdiag Thomas
    equals the dense block Thomas and a dense direct solve."""
    g = golden("thomas.npz")
    d, su, sb, r = g["diag_small_diag"], g["diag_small_sup"], g["diag_small_sub"], g["diag_small_rhs"]
    nz, ni = r.shape
    Mx = np.zeros((nz * ni, nz * ni))
    for j in range(nz):
        Mx[j * ni:(j + 1) * ni, j * ni:(j + 1) * ni] = d[j]
    for j in range(nz - 1):
        Mx[j * ni:(j + 1) * ni, (j + 1) * ni:(j + 2) * ni] = np.diag(su[j])
        Mx[(j + 1) * ni:(j + 2) * ni, j * ni:(j + 1) * ni] = np.diag(sb[j])
    x_dense = np.linalg.solve(Mx, r.reshape(-1)).reshape(nz, ni)
    close(orc.block_thomas(d, su, sb, r), x_dense, rtol=1e-12, floor=1e-12)


def test_contract_functions():
    g = golden("contract.npz")
    y, mix, sm, ng = oc.clip(g["sol"], g["ymix_old"], 1e-22, 0.0, -1.0, gas_mask=g["gas"])
    close(y, g["clip_gas_y"], 0.0); close(mix, g["clip_gas_mix"], 0.0)
    close(sm, g["clip_gas_small"], 0.0); close(ng, g["clip_gas_nega"], 0.0)
    y2, mix2, sm2, ng2 = oc.clip(g["sol"], g["ymix_old"], 1e-22, 0.0, -1.0)
    close(y2, g["clip_all_y"], 0.0); close(mix2, g["clip_all_mix"], 0.0)
    close(oc.aggregate_delta(y, g["delta"], g["ymix_old"], 1e-22, 1e-1), g["agg"], 0.0)
    close(oc.aggregate_delta(y, g["delta"], g["ymix_old"], 1e-22, 1e-1, True, g["cz"]), g["agg_bot"], 0.0)
    dtn = [oc.step_size(dt, dl, 0.2, 0.5, 2.0, 1e-14, 1e-2) for dt, dl in zip(g["dts"], g["deltas"])]
    close(dtn, g["dt_next"], 0.0)
    close(oc.atom_loss(np.abs(g["sol"]), g["compo"], g["atom_ini"]), g["atom_loss"], 1e-15)


def check_body_state(got, ref, rtol):
    """Counters and decisions exact; floating state within ``rtol``."""
    for f in ("accept_count", "retry_count", "nega_count", "loss_count", "delta_count"):
        assert int(got[f]) == int(ref[f]), (f, got[f], ref[f])
    for f in BODY_FIELDS:
        if f.endswith("_count"):
            continue
        close(got[f], ref[f], rtol, floor=1e-30)


def test_loop_body_attempts():
    """The restated loop body against one attempt of the reference runner
    (`outer_loop.py:715-1100`) per case, and a chain of eight attempts."""
    net, atm, compo, atom_ini, k, params, cases = golden_body()
    for name, c in cases.items():
        p, kw = body_kwargs(c, params)
        s = dict(c["inp"])
        for i in range(len(c["hist"])):
            prev = (s["accept_count"], s["retry_count"])
            s = oc.attempt(s, k, atm, net, compo, atom_ini, p, **kw)
            assert s["accept_count"] - prev[0] == c["hist"][i][0], (name, i)
        check_body_state(s, c["out"], 1e-13)


def test_convergence_chain():
    """Ring buffer, longdy / longdydt, stall detector and the loop condition
    against 40 attempts of the reference runner (``tests/golden/conv.npz``)."""
    net, atm, compo, atom_ini, k, params, cases = golden_body()
    g = golden("conv.npz")
    cp = {kk[len("conv_param_"):]: g[kk].item() for kk in g if kk.startswith("conv_param_")}
    p = dict(params, **cp)
    p.update(runtime=1e30, count_max=10 ** 6, conv_step=4, use_adapt_rtol=False)
    al = g["conv_in_atom_loss"]
    s = dict(y=g["conv_in_y"], y_prev=g["conv_in_y"], ymix=g["conv_in_ymix"], dt=1e-6, t=0.0, delta=0.0,
             accept_count=0, retry_count=0, atom_loss=al, atom_loss_prev=al, nega_count=0, loss_count=0,
             delta_count=0, small_y=1.5, nega_y=2.5, rtol=0.05, loss_criteria=1e-3, longdy=1.0, longdydt=1.0,
             longdy_seen_min=np.inf, count_since_new_min=0)
    nz, ni = s["y"].shape
    ring_y, ring_t = np.zeros((4, nz, ni)), np.zeros(4)
    for a in range(int(g["conv_n"])):
        s = oc.attempt(s, k, atm, net, compo, atom_ini, p)
        s.update(oc.conv_update(s, ring_y, ring_t, atm["M"], p, do_accept=s["_accept"] or s["_force"]))
        for f in ("accept_count", "retry_count", "count_since_new_min"):
            assert int(s[f]) == int(g["conv_" + f][a]), (a, f)
        for f in ("t", "dt", "longdy", "longdydt", "longdy_seen_min"):
            close(s[f], g["conv_" + f][a], 1e-12, floor=1e-300)
        assert oc.loop_continues(s, p, float(g["conv_slope_min"])) == bool(g["conv_cond"][a]), a
    close(ring_y, g["conv_y_ring"], 1e-12, floor=1e-30)
    close(ring_t, g["conv_t_ring"], 1e-12)


def _ph(g):
    return {k[3:]: (g[k].item() if g[k].ndim == 0 else g[k]) for k in g if k.startswith("ph_")}


def test_photo_kernels():
    g = golden("photo.npz")
    ph = _ph(g)
    close(op.compute_tau(g["y"], g["dz"], ph), g["tau"], 1e-14)
    for tag, ag0 in (("ag0", 0.0), ("ag3", 0.3)):
        p2 = dict(ph, ag0=ag0)
        aflux, sflux, dd, du = op.compute_flux(g["tau"], g["ymix"], p2, g["dflux_u_prev"])
        close(aflux, g[f"{tag}_aflux"], 1e-13); close(sflux, g[f"{tag}_sflux"], 1e-13)
        close(dd, g[f"{tag}_dflux_d"], 1e-13); close(du, g[f"{tag}_dflux_u"], 1e-13)
    Jb, JbT = op.compute_J(g["ag0_aflux"], ph)
    close(Jb, g["J_br"], 1e-13); close(JbT, g["J_br_T"], 1e-13)
    kn = op.update_k_with_J(g["k"], g["J_br"], g["J_br_T"], ph["branch_re_idx"], g["active"],
                            ph["branch_T_re_idx"], g["active_T"], 0.5)
    close(kn, g["k_new"], 0.0)


def test_synthetic_network_balances_elements():
    syn = load_pkg("synthetic")
    net = syn.make_network(0, 69, 700)
    t = net.tables
    assert t.ni == 69 and t.nr == 1400
    for r in range(1, t.nr + 1):
        lhs = sum(net.compo[i] * s for i, s in zip(t.reactant_idx[r], t.reactant_stoich[r]) if i < t.ni)
        rhs = sum(net.compo[i] * s for i, s in zip(t.product_idx[r], t.product_stoich[r]) if i < t.ni)
        np.testing.assert_array_equal(lhs, rhs)


def _chain(g):
    NT = load_pkg("network").NetworkTables
    net = NT(species=("A", "B"), ni=2, nr=6, reactant_idx=g["chain_r_idx"], product_idx=g["chain_p_idx"],
             reactant_stoich=g["chain_r_st"], product_stoich=g["chain_p_st"], is_three_body=g["chain_three"],
             is_photo=np.zeros(7, bool))
    nz, ni = 4, 2
    atm = dict(Kzz=np.full(nz - 1, 1e-2), Dzz=np.full((nz - 1, ni), 1e-3), dzi=np.full(nz - 1, 1.0),
               vz=np.zeros(nz - 1), Hpi=np.full(nz - 1, 1.0), Ti=np.full(nz - 1, 1500.0), Tco=np.full(nz, 1500.0),
               g=np.full(nz, 1.0), ms=np.full(ni, 1.0), alpha=np.zeros(ni), M=np.full(nz, 1.0),
               vm=np.zeros((nz, ni)), vs=np.zeros((nz - 1, ni)), top_flux=np.zeros(ni), bot_flux=np.zeros(ni),
               bot_vdep=np.zeros(ni), gas_indx_mask=np.ones(ni, dtype=bool), use_vm_mol=False,
               use_settling=False, use_topflux=False, use_botflux=False)
    k = np.zeros((7, nz))
    k[1], k[3], k[5] = 1.0, 0.5, 0.3
    return net, atm, k


def test_adjoint_known_answer_chain():
    """Reference tests/test_steady_state_grad.py: Newton steady state of the
    open chain (well mixed: [A]=k1/k3=2, [B]=k1/k5=3.33), the implicit gradient
    equals the reference's _ss_bwd and central finite differences."""
    from oracle import adjoint as oa
    g = golden("adjoint.npz")
    net, atm, k = _chain(g)
    y0 = np.zeros((4, 2))
    y0[:, 0], y0[:, 1] = 2.0, 3.3
    y, _ = oa.newton_steady_state(y0, k, atm, net)
    close(y, g["chain_y"], 1e-10)
    np.testing.assert_allclose(y[:, 0], 2.0, rtol=1e-2)
    np.testing.assert_allclose(y[:, 1], 1.0 / 0.3, rtol=1e-2)
    lam, cot = oa.ss_bwd(y, k, atm, net, g["chain_v"])
    close(cot["k_arr"], g["chain_gk"], 1e-10, floor=1e-12)
    eps = 1e-6
    fd = np.zeros_like(k)
    for i, z in [(i, z) for i in range(7) for z in range(4) if k[i, z] > 0]:
        kp, km = k.copy(), k.copy()
        kp[i, z] += eps
        km[i, z] -= eps
        yp, _ = oa.newton_steady_state(y0, kp, atm, net)
        ym, _ = oa.newton_steady_state(y0, km, atm, net)
        fd[i, z] = (np.sum(yp[:, 1] ** 2) - np.sum(ym[:, 1] ** 2)) / (2 * eps)
    assert np.max(np.abs(cot["k_arr"] - fd)) / np.max(np.abs(fd)) < 5e-4


def test_adjoint_k_gradient_matches_reference():
    from oracle import adjoint as oa
    g = golden("adjoint.npz")
    net = load_pkg("network").parse_network_text(str(g["case_net_text"]))
    from conftest import ATM_KEYS, FLAG_KEYS
    atm = {kk: g["case_atm_" + kk] for kk in ATM_KEYS}
    atm.update({kk: bool(g["case_atm_" + kk]) for kk in FLAG_KEYS})
    lam, cot = oa.ss_bwd(g["case_y"], g["case_k"], atm, net, g["case_v"])
    scale = k_gradient_scale(g["case_y"], atm["M"], lam, net)
    assert np.all(np.abs(cot["k_arr"] - g["case_gk"]) <= 1e-12 * scale)


def k_gradient_scale(y, M, lam, net):
    """Rounding scale of d(lam . f)/dk[r, z]: P'[z, r] * sum_s |st * lam| (the
    gradient is a sum of signed terms that can cancel)."""
    Pp = orc.rates(y, M, np.ones((net.nr + 1, y.shape[0])), net)          # [nz, nr+1]
    lp = np.concatenate([np.abs(lam), np.zeros((y.shape[0], 1))], axis=1)
    s = (np.abs(net.product_stoich)[None] * lp[:, net.product_idx]).sum(2) + \
        (np.abs(net.reactant_stoich)[None] * lp[:, net.reactant_idx]).sum(2)
    return (np.abs(Pp) * s).T


def _rates_case():
    g = golden("rates.npz")
    net = load_pkg("network").parse_network_text(str(g["net_text"]))
    return g, net


def test_rate_build_matches_reference():
    """Reference rates.py / gibbs.py (tests/golden/rates.npz): this package's
    parser reads the same rate columns and flags, and the oracle reproduces
    every stage bit for bit; its complex-step dk/dT agrees with central
    differences (h = 1e-4 K) to their truncation error, away from the
    branch switches at 200, 277.5, 300 and 1000 K."""
    from oracle import rates as orr
    g, net = _rates_case()
    for f in ("a", "n", "E", "a_inf", "n_inf", "E_inf", "is_forward", "has_kinf", "is_special", "is_conden",
              "is_radiative", "is_photo", "is_ion"):
        np.testing.assert_array_equal(getattr(net, f), g["net_" + f], err_msg=f)
    assert net.stop_rev_indx == int(g["stop_rev_indx"])
    T, M, c, rm = g["T"], g["M"], g["coeffs"], list(g["remove"])
    kf = orr.compute_forward_k(net, T, M)
    np.testing.assert_array_equal(kf, g["k_fwd"])
    np.testing.assert_array_equal(orr.apply_lowT_caps(net, kf, T, M), g["k_caps"])
    gs = orr.gibbs_sp_vector(c, T)
    np.testing.assert_array_equal(gs, g["g"])
    K = orr.K_eq_array(net, gs, T)
    np.testing.assert_array_equal(K, g["K"])
    np.testing.assert_array_equal(orr.fill_reverse_k(net, kf, K), g["k_nocap"])
    k = orr.build_rate_array(net, c, T, M, lowT_caps=True, remove_list=rm)
    np.testing.assert_array_equal(k, g["k_all"])
    d = orr.dk_dT(net, c, T, M, lowT_caps=True, remove_list=rm)
    h = 1e-4
    fd = (orr.build_rate_array(net, c, T + h, M, True, rm) - orr.build_rate_array(net, c, T - h, M, True, rm)) / (2 * h)
    ok = np.all([np.abs(T - t) > 1e-3 for t in (200.0, 277.5, 300.0, 1000.0)], axis=0)
    scale = np.maximum(np.abs(fd[:, ok]), 1e-12 * np.abs(k[:, ok]) + 1e-300)
    assert np.max(np.abs(d[:, ok] - fd[:, ok]) / scale) < 1e-4
