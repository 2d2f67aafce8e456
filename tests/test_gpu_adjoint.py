"""Implicit steady-state adjoint on the GPU against the reference-generated
fixture (its own _ss_bwd) and the oracle.

Tolerances: the k-gradient is a sum of signed terms that can cancel, so each
entry must lie within 1e-10 of its rounding scale P'[r,z] sum|st*lambda|; the
other cotangents within 1e-10 relative to the largest entry of their leaf;
lambda by its normwise backward error (<= 1e-12) on J_y^T lambda = v.
"""
import numpy as np
import pytest
import torch

from conftest import ATM_KEYS, FLAG_KEYS, golden, load_pkg
from oracle import adjoint as oa
from test_oracle_golden import _chain, k_gradient_scale

pytestmark = pytest.mark.gpu
chem = load_pkg("chem")
jstep = load_pkg("jax_step")
ssg = load_pkg("steady_state_grad")
syn = load_pkg("synthetic")


def normwise(a, b):
    return float(np.max(np.abs(np.asarray(a) - b)) / max(np.max(np.abs(b)), 1e-300))


def test_chain_gradient_matches_reference():
    g = golden("adjoint.npz")
    net, atm, k = _chain(g)
    dn = chem.to_device(net)
    cot = ssg.implicit_cotangents(g["chain_y"], k, jstep.atm_from_dict(atm), dn, g["chain_v"])
    assert normwise(cot["k_arr"].cpu().numpy(), g["chain_gk"]) <= 1e-10
    assert int(cot["status"].cpu()[0]) == 0


def test_k_gradient_matches_reference_case():
    g = golden("adjoint.npz")
    net = load_pkg("network").parse_network_text(str(g["case_net_text"]))
    atm = {kk: g["case_atm_" + kk] for kk in ATM_KEYS}
    atm.update({kk: bool(g["case_atm_" + kk]) for kk in FLAG_KEYS})
    dn = chem.to_device(net)
    cot = ssg.implicit_cotangents(g["case_y"], g["case_k"], jstep.atm_from_dict(atm), dn, g["case_v"])
    lam_ref, _ = oa.ss_bwd(g["case_y"], g["case_k"], atm, net, g["case_v"])
    scale = k_gradient_scale(g["case_y"], atm["M"], lam_ref, net)
    assert np.all(np.abs(cot["k_arr"].cpu().numpy() - g["case_gk"]) <= 1e-10 * scale)


@pytest.mark.parametrize("transport", [dict(moldiff=True, fluxes=True),
                                       dict(moldiff=True, advection=True, fluxes=True)])
def test_all_leaves_batched_against_oracle(transport):
    """Every SteadyStateInputs leaf (steady_state_grad.py:36-59): lambda and the
    cotangents against the oracle's autograd VJP at the GPU's lambda. The first
    transport set exercises the gravity / thermal-diffusion leaves (Hpi, Ti,
    Tco, g, ms, alpha), the second the advection and settling leaves (vz, vm,
    vs), which replace the gravity term."""
    net = syn.make_network(44, 30, 185, n_three_body=20)
    dn = chem.to_device(net.tables)
    cases = [syn.make_case(seed=50 + b, net=net, nz=24, mild=True, k_range=(-40.0, 4.0), **transport)
             for b in range(3)]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    V = np.random.default_rng(5).normal(0.0, 1.0, Y.shape) / np.abs(Y)
    cot = ssg.implicit_cotangents(Y, K, jstep.atm_from_dict(A), dn, V)
    for b, c in enumerate(cases):
        lam, _ = oa.ss_bwd(c.y, c.k, c.atm, net.tables, V[b])
        lam_g = cot["lambda"][b].cpu().numpy()
        # lambda solves J_y^T lambda = v: its normwise backward error is at
        # rounding level (the advection terms make the system less well
        # conditioned, so the forward difference to the oracle is only loose)
        diag, sup, sub = oa.jacobian_blocks(c.y, c.k, c.atm, net.tables)
        res = np.einsum("zji,zj->zi", diag, lam_g)
        res[:-1] += sub * lam_g[1:]
        res[1:] += sup * lam_g[:-1]
        res -= V[b]
        normA = max(np.abs(diag).sum(axis=1).max(), 1.0)
        assert np.abs(res).max() / (normA * np.abs(lam_g).max() + np.abs(V[b]).max()) <= 1e-12
        assert normwise(lam_g, lam) <= 1e-8
        # the VJP kernels given the GPU's lambda
        ref = oa.vjp_from_lambda(c.y, c.k, c.atm, net.tables, lam_g)
        scale = k_gradient_scale(c.y, c.atm["M"], lam_g, net.tables)
        assert np.all(np.abs(cot["k_arr"][b].cpu().numpy() - ref["k_arr"]) <= 1e-12 * scale)
        for leaf in oa.LEAVES:
            if leaf == "k_arr":
                continue
            got = cot[leaf][b].cpu().numpy()
            assert got.shape == np.shape(ref[leaf]), leaf
            assert normwise(got, ref[leaf]) <= 1e-10, (leaf, normwise(got, ref[leaf]))
        # the Kzz cotangent by differentiating the stencil equals the hand-derived one
        assert normwise(cot["Kzz_transport"][b].cpu().numpy(), cot["Kzz"][b].cpu().numpy()) <= 1e-10


def test_autograd_function_chain():
    """torch.autograd through DifferentiableSteadyState gives the reference
    custom_vjp gradient of sum(y[:,1]**2) (tests/test_steady_state_grad.py)."""
    g = golden("adjoint.npz")
    net, atm, k = _chain(g)
    dn = chem.to_device(net)
    kt = torch.as_tensor(k, device="cuda").requires_grad_(True)
    y = torch.as_tensor(g["chain_y"], device="cuda")
    ys = ssg.differentiable_steady_state(kt, y, jstep.atm_from_dict(atm), dn)
    (ys[:, 1] ** 2).sum().backward()
    assert normwise(kt.grad.cpu().numpy(), g["chain_gk"]) <= 1e-10


def test_residual_gate():
    g = golden("adjoint.npz")
    net, atm, k = _chain(g)
    dn = chem.to_device(net)
    r = ssg.validate_steady_state_solution(g["chain_y"], k, jstep.atm_from_dict(atm), dn)
    assert r < 1e-9
    with pytest.raises(ValueError):
        ssg.validate_steady_state_solution(g["chain_y"] * 1.5, k, jstep.atm_from_dict(atm), dn)


def test_temperature_gradient_through_rates_and_transport():
    """dL/dT per layer = the Tco leaf + the interface-temperature leaf (Ti the
    mean of its two layers) + sum_r g_k dk_r/dT (vb_rates' dual-number dk/dT),
    against the complex-step derivative of phi(T) = -lambda . f(y, k(T),
    atm(T)) on the oracle, with lambda from the GPU adjoint: the adjoint
    identity g_theta = -lambda . df/dtheta holds for any lambda. Network with
    Arrhenius and Lindemann rates and NASA-9 reverse rates (12 species, 30 +
    30 reactions), molecular diffusion with thermal diffusion on, 10 layers
    from 800 to 2000 K.

    The block-tridiagonal system is singular to working precision (condition
    ~1e36: element balance makes each layer's atom-count vectors near-null
    vectors of J^T, broken only by transport), so lambda carries a large
    solver-dependent null-space component that cancels inside every
    reaction's cotangent. The tolerance is therefore stated against the
    rounding scale of the contraction, the sum of the magnitudes of all its
    terms (per reaction |dk_r/dT| |rate_r/k_r| sum_i |nu_ir lambda_i|, per
    transport element |lambda_i d diff_i/dT|): 1e-12 of it. Two CPU
    evaluations of the same contraction in different orders agree to ~1e-17
    of that scale while differing by up to 100 % of max |dL/dT|."""
    from types import SimpleNamespace
    from oracle import rates as orr
    rates = load_pkg("rates")
    net_tab = load_pkg("network").parse_network_text(
        syn.make_rate_network(3, ni=12, n_fwd=30, n_kinf=6, n_nokinf=3, n_photo=0, special=False))
    coeffs = syn.make_nasa9(3, net_tab.ni)
    rng = np.random.default_rng(3)
    ms = rng.uniform(2.0, 60.0, net_tab.ni)
    atm, extra = syn.make_atmosphere(3, SimpleNamespace(tables=net_tab, ms=ms), nz=10, moldiff=True)
    T, M = atm["Tco"].copy(), atm["M"]
    assert np.all(np.abs(T - 1000.0) > 1.0)            # away from the NASA-9 branch switch
    k = orr.build_rate_array(net_tab, coeffs, T, M)
    y = extra["y"]
    v = rng.normal(0.0, 1.0, y.shape) / np.abs(y)
    dn = chem.to_device(net_tab)
    cot = ssg.implicit_cotangents(y, k, jstep.atm_from_dict(atm), dn, v)
    _, dkdT = rates.RateTables(net_tab, coeffs)(T, M, with_dkdT=True)
    gT = ssg.temperature_cotangent(cot, dkdT).cpu().numpy()
    lam = cot["lambda"].cpu().numpy()

    from oracle import ros2 as oros2

    def f_of(Tz):
        a = dict(atm, Tco=Tz, Ti=0.5 * (Tz[1:] + Tz[:-1]))
        return oa.residual(y, orr.build_rate_array(net_tab, coeffs, Tz, M), a, net_tab)

    def diff_of(Tz):
        return oros2.diffusion(y, dict(atm, Tco=Tz, Ti=0.5 * (Tz[1:] + Tz[:-1])))[0]

    h, eye = 1e-30, np.eye(10)
    g_cs = np.array([-np.sum(lam * np.imag(f_of(T + 1j * h * eye[z])) / h) for z in range(10)])
    lam_p = np.concatenate([lam, np.zeros((10, 1))], axis=1)          # slot ni: no species
    nu_lam = (np.abs(net_tab.reactant_stoich[None] * lam_p[:, net_tab.reactant_idx]).sum(-1)
              + np.abs(net_tab.product_stoich[None] * lam_p[:, net_tab.product_idx]).sum(-1))
    per_k = oros2.rates(y, M, np.ones_like(k), net_tab)                # rate_r / k_r
    s_chem = np.sum(np.abs(orr.dk_dT(net_tab, coeffs, T, M).T) * np.abs(per_k) * nu_lam, axis=1)
    s_tr = np.array([np.sum(np.abs(lam * np.imag(diff_of(T + 1j * h * eye[z])) / h)) for z in range(10)])
    scale = float(np.max(s_chem + s_tr))
    err = np.max(np.abs(gT - g_cs)) / scale
    print(f"dL/dT vs complex step: {err:.2e} of the contraction's rounding scale")
    assert err <= 1e-12, (gT, g_cs, scale)


def test_adjoint_on_unconverged_stiff_states():
    """Two config-4-shaped atmospheres (ni=69, 700 + 700 Arrhenius / Lindemann
    reactions with NASA-9 reverse rates plus 40 photolysis rows, nz=120,
    molecular diffusion and boundary fluxes on) at their unconverged seeded
    states, where the block system is singular to working precision
    (diagonal blocks of condition 1e22-1e33). lambda itself is not determined
    there, but the solve must stay finite, report no status bit, and be
    backward stable: ||J^T lambda - v|| / (||J^T|| ||lambda|| + ||v||) below
    1e-14 against the oracle's Jacobian blocks (the reference algorithm, LU +
    substitution, reaches ~1e-24 here). Eliminating on the transposed blocks
    for these transposed solves gave a zero pivot and no finite lambda."""
    from types import SimpleNamespace
    from oracle import rates as orr
    net_tab = load_pkg("network").parse_network_text(
        syn.make_rate_network(0, ni=69, n_fwd=700, n_kinf=60, n_nokinf=20, n_photo=40, special=False))
    coeffs = syn.make_nasa9(0, net_tab.ni)
    ms = np.random.default_rng(0).uniform(2.0, 60.0, net_tab.ni)
    dn = chem.to_device(net_tab)
    for b in range(2):
        atm, extra = syn.make_atmosphere((b,), SimpleNamespace(tables=net_tab, ms=ms), nz=120, moldiff=True,
                                         fluxes=True)
        k = orr.build_rate_array(net_tab, coeffs, atm["Tco"], atm["M"])
        y = extra["y"]
        v = np.random.default_rng(5 + b).normal(0.0, 1.0, y.shape)
        cot = ssg.implicit_cotangents(y, k, jstep.atm_from_dict(atm), dn, v)
        assert int(cot["status"].reshape(-1)[0]) == 0
        for name, val in cot.items():
            if name != "status":
                assert bool(torch.isfinite(val).all()), name
        lam = cot["lambda"].cpu().numpy()
        diag, sup, sub = oa.jacobian_blocks(y, k, atm, net_tab)
        r = np.einsum("zji,zj->zi", diag, lam)          # J_j^T lambda_j
        r[:-1] += sub * lam[1:]
        r[1:] += sup * lam[:-1]
        r -= v
        norm_jt = max(np.abs(diag).sum(axis=1).max(), 1.0)
        bwd = np.abs(r).max() / (norm_jt * np.abs(lam).max() + np.abs(v).max())
        print(f"atmosphere {b}: backward error {bwd:.2e}, max |lambda| {np.abs(lam).max():.2e}")
        assert bwd <= 1e-14, bwd

