"""CUDA path against the oracle and the reference-generated fixtures.

Tolerances (FP64 path):
* chemistry RHS and analytic Jacobian are gathered in the reference's
  summation order; they are bit-identical except where NumPy's ``pow(y, 2)``
  and the GPU's ``y*y`` round differently, so each entry must lie within
  ``4 eps * sum|terms|`` (the rounding bound of its gather) and at least 99% of
  entries must be bit-identical; diffusion coefficients are bit-identical;
* Ros2 step outputs: ``|sol - ref| <= 1e-10 * max(|ref|, 1e-30)`` and, since
  the error estimate is consumed as ``delta / sol`` (reference
  `outer_loop.py:227-250`), ``|delta - ref| <= 1e-10 * max(|sol_ref|, 1e-30)``;
* block solver: ``1e-10`` relative (floor 1e-12) against the reference solver.
The step comparisons use well-conditioned draws (order-scaled rate constants);
the stiff draws of the benchmark configurations make a single step
ill-conditioned (sensitivity > 1e10), so there the step is checked through
its exactly-reproducible parts and the normwise backward error of the solve.
"""
import numpy as np
import pytest
import torch

from conftest import STEP_CASES, golden, golden_step, load_pkg
from oracle import ros2 as orc

pytestmark = pytest.mark.gpu

chem = load_pkg("chem")
jstep = load_pkg("jax_step")
solver = load_pkg("solver")
syn = load_pkg("synthetic")


def rel_err(a, b, floor=1e-30):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor), initial=0.0))


def check_step(sol, delta, sol_ref, delta_ref, tol=1e-10):
    sol, delta = np.asarray(sol), np.asarray(delta)
    e_sol = rel_err(sol, sol_ref)
    e_del = float(np.max(np.abs(delta - delta_ref) / np.maximum(np.abs(sol_ref), 1e-30)))
    assert e_sol <= tol, f"sol rel err {e_sol:.3e}"
    assert e_del <= tol, f"delta err {e_del:.3e}"
    return e_sol, e_del


def atm_of(atm):
    return jstep.atm_from_dict(atm)


@pytest.mark.parametrize("name", STEP_CASES + ["stiff"])
def test_chem_bit_identical_to_reference(name):
    net, atm, y, k, dt, fm, g = golden_step(name)
    dn = chem.to_device(net)
    rhs = chem.chem_rhs(y, atm["M"], k, dn).cpu().numpy()
    jac = chem.chem_jac_analytical(y, atm["M"], k, dn).cpu().numpy()
    check_gather(rhs, g["rhs"], orc.chem_rhs_abs(y, atm["M"], k, net))
    check_gather(jac, g["jac"], orc.chem_jac_abs(y, atm["M"], k, net))


EPS = np.finfo(np.float64).eps


def check_gather(a, ref, abs_sum):
    assert np.all(np.abs(a - ref) <= 4 * EPS * abs_sum), float(np.max(np.abs(a - ref) / np.maximum(abs_sum, 1e-300)))
    assert np.mean(a == ref) >= 0.99, np.mean(a == ref)


@pytest.mark.parametrize("name", ["plain", "moldiff", "full", "fixmask", "medium"])
def test_diffusion_bit_identical_to_oracle(name):
    net, atm, y, k, dt, fm, g = golden_step(name)
    diff, diag_d, sup, sub = jstep.diffusion(y, atm_of(atm))
    grav = orc.compute_diff_grav(atm)
    co = orc.build_diff_coeffs(y, atm, grav)
    ref_diff = orc.apply_diffusion(y, *co[:6], atm)
    A_e, B_e, C_e, A_m, B_m, C_m, _ = co
    ref_dd = A_e[:, None] + A_m
    if atm["use_botflux"]:
        ref_dd[0] = ref_dd[0] + (-atm["bot_vdep"] / atm["dzi"][0])
    np.testing.assert_array_equal(diff.cpu().numpy(), ref_diff)
    np.testing.assert_array_equal(diag_d.cpu().numpy(), ref_dd)
    np.testing.assert_array_equal(sup.cpu().numpy(), B_e[:-1, None] + B_m[:-1])
    np.testing.assert_array_equal(sub.cpu().numpy(), C_e[1:, None] + C_m[1:])


@pytest.mark.parametrize("name", STEP_CASES)
def test_ros2_step_matches_reference_fixture(name):
    net, atm, y, k, dt, fm, g = golden_step(name)
    dn = chem.to_device(net)
    sol, delta = jstep.jax_ros2_step(y, k, dt, atm_of(atm), dn, fix_mask=fm)
    check_step(sol.cpu(), delta.cpu(), g["sol"], g["delta"])


@pytest.mark.parametrize("flags", [dict(), dict(moldiff=True), dict(moldiff=True, advection=True, fluxes=True)])
def test_ros2_step_config0_size(flags):
    """ni=69, 700+700 reactions, nz=120 (the config-0 shape), well-conditioned draw."""
    case = syn.make_case(seed=31, mild=True, k_range=(-40.0, 4.0), **flags)
    sol_ref, delta_ref = orc.ros2_step(case.y, case.k, case.dt, case.atm, case.net.tables)
    dn = chem.to_device(case.net.tables)
    sol, delta = jstep.jax_ros2_step(case.y, case.k, case.dt, atm_of(case.atm), dn)
    check_step(sol.cpu(), delta.cpu(), sol_ref, delta_ref)


def test_ros2_step_sncho_size_with_fix_mask():
    """ni=89 with sulfur, 2000 reactions, nz=150 (the config-3 shape), fix_mask."""
    case = syn.make_case(seed=33, ni=89, n_fwd=1000, nz=150, elements=("C", "H", "O", "N", "S"),
                         mild=True, k_range=(-45.0, 4.0), moldiff=True, fluxes=True, n_three_body=40)
    fm = np.random.default_rng(3).random(case.y.shape) < 0.02
    sol_ref, delta_ref = orc.ros2_step(case.y, case.k, case.dt, case.atm, case.net.tables, fix_mask=fm)
    dn = chem.to_device(case.net.tables)
    sol, delta = jstep.jax_ros2_step(case.y, case.k, case.dt, atm_of(case.atm), dn, fix_mask=fm)
    check_step(sol.cpu(), delta.cpu(), sol_ref, delta_ref)


def test_batched_step_equals_single_steps():
    """vmap semantics (reference tests/test_vmap_step.py): a batch of different
    atmospheres gives exactly the per-atmosphere results."""
    net = syn.make_network(41, 30, 185)
    dn = chem.to_device(net.tables)
    cases = [syn.make_case(seed=40 + b, net=net, nz=24, mild=True, k_range=(-40.0, 4.0), moldiff=True)
             for b in range(3)]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    dts = np.array([1e-6, 1e-4, 1e-8])
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    sol_b, delta_b = jstep.jax_ros2_step(Y, K, dts, atm_of(A), dn)
    for b, c in enumerate(cases):
        s1, d1 = jstep.jax_ros2_step(c.y, c.k, dts[b], atm_of(c.atm), dn)
        assert torch.equal(sol_b[b], s1) and torch.equal(delta_b[b], d1)
        sref, dref = orc.ros2_step(c.y, c.k, dts[b], c.atm, c.net.tables)
        check_step(s1.cpu(), d1.cpu(), sref, dref)


def test_batch_beyond_sm_count():
    """More atmospheres than SMs (the factor then runs two CTAs per SM with a
    different warp layout): sampled atmospheres against the oracle and against
    the same atmosphere stepped alone."""
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    B = n_sm + 4
    net = syn.make_network(43, 69, 700)
    dn = chem.to_device(net.tables)
    cases = [syn.make_case(seed=(900 + b,), net=net, nz=8, mild=True, k_range=(-40.0, 4.0)) for b in range(B)]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    dts = np.full(B, 1e-6)
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    sol_b, delta_b = jstep.jax_ros2_step(Y, K, dts, atm_of(A), dn)
    sol_b, delta_b = sol_b.cpu().numpy(), delta_b.cpu().numpy()
    for b in (0, 1, n_sm - 1, n_sm, B - 1):
        c = cases[b]
        sref, dref = orc.ros2_step(c.y, c.k, dts[b], c.atm, c.net.tables)
        check_step(sol_b[b], delta_b[b], sref, dref)
        s1, d1 = jstep.jax_ros2_step(c.y, c.k, dts[b], atm_of(c.atm), dn)
        check_step(sol_b[b], delta_b[b], s1.cpu().numpy(), d1.cpu().numpy())


def test_block_thomas_reference_systems():
    g = golden("thomas.npz")
    x = solver.block_thomas_diag_offdiag(g["diag_small_diag"], g["diag_small_sup"], g["diag_small_sub"],
                                         g["diag_small_rhs"]).cpu().numpy()
    assert rel_err(x, g["diag_small_x"], 1e-12) <= 1e-10
    rng = np.random.default_rng(7)
    rng.standard_normal((8, 5, 5)); rng.standard_normal((7, 5)); rng.standard_normal((7, 5))
    rng.standard_normal((8, 5))
    d2 = rng.standard_normal((120, 93, 93)) + 1e10 * np.eye(93)
    su2 = rng.standard_normal((119, 93)) * 1e-3
    sb2 = rng.standard_normal((119, 93)) * 1e-3
    r2 = rng.standard_normal((120, 93))
    x2 = solver.block_thomas_diag_offdiag(d2, su2, sb2, r2).cpu().numpy()
    assert rel_err(x2, g["diag_big_x"], 1e-12) <= 1e-10


def test_block_thomas_transposed_solve():
    rng = np.random.default_rng(2)
    nz, ni = 16, 8
    diag = rng.standard_normal((nz, ni, ni))
    diag = diag + (5.0 + np.abs(diag).sum(axis=2))[:, :, None] * np.eye(ni)[None]
    su = 0.1 * rng.standard_normal((nz - 1, ni))
    sb = 0.1 * rng.standard_normal((nz - 1, ni))
    rhs = rng.standard_normal((nz, ni))
    f = solver.factor_block_thomas_diag_offdiag(diag, su, sb)
    xT = solver.solve_block_thomas_diag_offdiag_T(f, rhs).cpu().numpy()
    ref = orc.block_thomas(np.transpose(diag, (0, 2, 1)), sb, su, rhs)
    assert rel_err(xT, ref, 1e-12) <= 1e-10
    x = solver.solve_block_thomas_diag_offdiag(f, rhs).cpu().numpy()
    assert rel_err(x, orc.block_thomas(diag, su, sb, rhs), 1e-12) <= 1e-10


def test_stiff_config0_inputs_backward_error():
    """The benchmark's config-0 draw (k log-uniform in [1e-40, 1e-8], dt=1e-6):
    the Jacobian matches within its gather bound; the block solve's normwise
    backward error ||A x - b|| / (||A|| ||x|| + ||b||) stays at rounding level."""
    case = syn.config0()
    dn = chem.to_device(case.net.tables)
    diag, sup_n, sub_n, rhs, _ = orc.lhs_blocks(case.y, case.k, case.dt, case.atm, case.net.tables)
    J = chem.chem_jac_analytical(case.y, case.atm["M"], case.k, dn).cpu().numpy()
    check_gather(J, orc.chem_jac(case.y, case.atm["M"], case.k, case.net.tables),
                 orc.chem_jac_abs(case.y, case.atm["M"], case.k, case.net.tables))
    x = solver.block_thomas_diag_offdiag(diag, sup_n, sub_n, rhs).cpu().numpy()
    nz = rhs.shape[0]
    res = np.einsum("zij,zj->zi", diag, x)
    res[:-1] += sup_n * x[1:]
    res[1:] += sub_n * x[:-1]
    res -= rhs
    normA = max(np.abs(diag).sum(axis=2).max(), 1.0)
    bwd = np.abs(res).max() / (normA * np.abs(x).max() + np.abs(rhs).max())
    assert np.isfinite(x).all()
    assert bwd < 1e-12, bwd


def test_status_flags():
    nz, ni = 4, 3
    diag = np.tile(np.eye(ni), (nz, 1, 1))
    diag[2] = 0.0                          # singular block
    su = np.zeros((nz - 1, ni))
    sb = np.zeros((nz - 1, ni))
    f = solver.factor_block_thomas_diag_offdiag(diag, su, sb)
    st = int(f.status.cpu()[0])
    assert st & 1, st


@pytest.mark.parametrize("ni,n_fwd", [(48, 400), (120, 900)])
def test_ros2_step_factor_shapes_mid_and_large(ni, n_fwd):
    """The factor's tile shapes for 33-64 species and for 97-128 species
    (the latter without the bulk prefetch of the next block), through the
    Ros2 step, well-conditioned draw."""
    net = syn.make_network(47, ni, n_fwd)
    case = syn.make_case(seed=48, net=net, nz=30, mild=True, k_range=(-40.0, 4.0), moldiff=True)
    sol_ref, delta_ref = orc.ros2_step(case.y, case.k, case.dt, case.atm, net.tables)
    dn = chem.to_device(net.tables)
    sol, delta = jstep.jax_ros2_step(case.y, case.k, case.dt, atm_of(case.atm), dn)
    check_step(sol.cpu(), delta.cpu(), sol_ref, delta_ref)


@pytest.mark.parametrize("ni", [48, 120])
def test_block_solves_fp64_and_mixed_mid_and_large(ni):
    """FP64 factor + solve and the mixed-precision (FP32 factor, FP64
    refinement) solve at the same two tile shapes, against the oracle's
    block Thomas at 1e-10."""
    rng = np.random.default_rng(ni)
    nz, B = 12, 3
    diag = rng.standard_normal((B, nz, ni, ni))
    diag = diag + (5.0 + np.abs(diag).sum(axis=3))[..., None] * np.eye(ni)
    su = 0.1 * rng.standard_normal((B, nz - 1, ni))
    sb = 0.1 * rng.standard_normal((B, nz - 1, ni))
    rhs = rng.standard_normal((B, nz, ni))
    x64 = solver.block_thomas_diag_offdiag(diag, su, sb, rhs).cpu().numpy()
    f = solver.factor_block_thomas_mixed(diag, su, sb)
    xm, passes = solver.solve_block_thomas_mixed(f, rhs, max_refine=3, tol=1e-14)
    xm = xm.cpu().numpy()
    assert int(f.status.cpu().max()) == 0
    for b in range(B):
        ref = orc.block_thomas(diag[b], su[b], sb[b], rhs[b])
        assert rel_err(x64[b], ref, 1e-12) <= 1e-10
        assert rel_err(xm[b], ref, 1e-12) <= 1e-10


@pytest.mark.parametrize("nz,kw", [(121, dict(moldiff=True, fluxes=True)), (24, dict(advection=True, fluxes=True)),
                                   (7, dict())])
def test_stage1_two_layers_per_cta_bit_identical(nz, kw):
    """The stage-1 assembly with two layers per CTA (VbTuning.stage1_layers =
    2) shares gather words between the layers but keeps each sum's order:
    the step is bit-identical to the one-layer kernel's (odd layer counts,
    bottom fluxes, a fix mask, a ragged batch included)."""
    at = load_pkg("autotune")
    net = syn.make_network(61, 30, 185)
    dn = chem.to_device(net.tables)
    cases = [syn.make_case(seed=(610 + b,), net=net, nz=nz, mild=True, k_range=(-40.0, 4.0), **kw) for b in range(3)]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    fm = np.random.default_rng(nz).random(Y.shape) < 0.03
    out = []
    for layers in (1, 2):
        at.set_tuning(dn, {"stage1_layers": layers})
        step = jstep.Ros2Step(dn, atm_of(A))
        s, d, st = step(Y, K, np.array([1e-6, 1e-4, 1e-8]), fix_mask=fm)
        out.append((s.clone(), d.clone(), st.clone()))
        rag = jstep.RaggedRos2Step(dn, [jstep.atm_from_dict(c.atm) for c in cases])
        y, k = rag.pack([c.y for c in cases], [c.k for c in cases])
        rs, rd, _ = rag(y, k, torch.as_tensor([1e-6, 1e-4, 1e-8], device="cuda"))
        out.append((rs.clone(), rd.clone(), None))
    at.set_tuning(dn, {})
    assert torch.equal(out[0][0], out[2][0]) and torch.equal(out[0][1], out[2][1])
    assert torch.equal(out[0][2], out[2][2]) and int(out[0][2].abs().sum()) == 0
    assert torch.equal(out[1][0], out[3][0]) and torch.equal(out[1][1], out[3][1])
    sref, dref = orc.ros2_step(cases[0].y, cases[0].k, 1e-6, cases[0].atm, net.tables, fix_mask=fm[0])
    check_step(out[2][0][0].cpu(), out[2][1][0].cpu(), sref, dref)
