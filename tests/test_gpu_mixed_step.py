"""The mixed-precision Ros2 step (``vb_ros2_step_mixed``): FP64 assembly,
row-equilibrated FP32 factor with TF32 tensor-core trailing updates, FP64
refinement of both stage solves, FP64 fallback.

Bounds:
* well-conditioned draws (order-scaled rate constants): status 0 (no
  fallback), every species within the metric's 1e-6 relative error of the
  FP64 oracle (``|sol - ref| <= 1e-6 max(|ref|, 1e-30)``, and delta against
  ``|sol_ref|``), and both stage solves at a normwise backward error below
  1e-12 against the oracle's FP64 system;
* the specified stiff draw: finite results, status 0 or VB_STATUS_REFINE_STALL
  (the FP64 fallback ran), both stage backward errors below 1e-11 (the bound
  of the FP64 kernels on these seeds: their inverse-based solves reach
  1.4e-12 on seed 10, tests/test_gpu_factor_variants.py).
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg
from oracle import ros2 as orc

pytestmark = pytest.mark.gpu

chem = load_pkg("chem")
jstep = load_pkg("jax_step")
syn = load_pkg("synthetic")

REL = 1e-6
BWD = 1e-12
BWD_STIFF = 1e-11
STALL = 4


def _batch(net, seeds, nz, mild, **kw):
    extra = dict(mild=True, k_range=(-40.0, 4.0)) if mild else {}
    cases = [syn.make_case(seed=(s,), net=net, nz=nz, **extra, **kw) for s in seeds]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    return cases, Y, K, np.array([c.dt for c in cases]), A


def _run(net, cases, Y, K, DT, A, **kw):
    dn = chem.to_device(net.tables)
    step = jstep.Ros2Step(dn, jstep.atm_from_dict(A), mixed=True, **kw)
    sol, delta, status = step(Y, K, DT)
    k1, k2 = step.stages()
    torch.cuda.synchronize()
    return (sol.cpu().numpy(), delta.cpu().numpy(), status.cpu().numpy().copy(), k1.cpu().numpy(),
            k2.cpu().numpy(), step.passes.cpu().numpy().copy())


_lib = load_pkg("_lib")


@pytest.fixture(params=[1, 0, 2], ids=["scalar_gj", "blocked_tf32", "pipelined_gj"])
def factor_kernel(request):
    _lib.check(_lib.lib().vb_set_factor_kernel(request.param), "vb_set_factor_kernel")
    yield request.param
    _lib.check(_lib.lib().vb_set_factor_kernel(1), "vb_set_factor_kernel")


@pytest.mark.parametrize("ni,n_fwd,nz", [(30, 185, 40), (69, 700, 120), (89, 1000, 60)])
def test_mixed_step_well_conditioned_within_1e6(factor_kernel, ni, n_fwd, nz):
    elements = ("C", "H", "O", "N", "S") if ni == 89 else ("C", "H", "O", "N")
    net = syn.make_network(80 + ni, ni, n_fwd, elements)
    cases, Y, K, DT, A = _batch(net, (1, 2, 3), nz, True, moldiff=True)
    sol, delta, st, k1, k2, passes = _run(net, cases, Y, K, DT, A)
    assert (st == 0).all(), st
    for b, c in enumerate(cases):
        sref, dref = orc.ros2_step(c.y, c.k, c.dt, c.atm, net.tables)
        rel = np.abs(sol[b] - sref) / np.maximum(np.abs(sref), 1e-30)
        e_del = np.max(np.abs(delta[b] - dref) / np.maximum(np.abs(sref), 1e-30))
        print(f"ni={ni} atmosphere {b}: passes {passes[b]}, max rel err {rel.max():.2e}, delta err {e_del:.2e}")
        assert rel.max() <= REL and e_del <= REL, (b, rel.max(), e_del)
        bwd = orc.stage_backward_errors(c.y, c.k, c.dt, c.atm, net.tables, k1[b], k2[b])
        assert max(bwd) < BWD, (b, bwd)


def test_mixed_step_stiff_draw_backward_errors():
    net = syn.make_network(0, 69, 700)
    cases, Y, K, DT, A = _batch(net, (0, 5, 10, 11), 120, False)
    sol, delta, st, k1, k2, passes = _run(net, cases, Y, K, DT, A)
    assert np.isfinite(sol).all() and np.isfinite(delta).all()
    assert ((st & ~STALL) == 0).all(), st
    for b, c in enumerate(cases):
        bwd = orc.stage_backward_errors(c.y, c.k, c.dt, c.atm, net.tables, k1[b], k2[b])
        print(f"stiff atmosphere {b}: status {st[b]}, passes {passes[b]}, backward errors {bwd[0]:.1e} {bwd[1]:.1e}")
        assert max(bwd) < BWD_STIFF, (b, bwd)


def test_mixed_step_without_refinement_falls_back():
    """max_refine = 0 on a draw FP32 cannot solve to the tolerance: every
    atmosphere stalls, takes the FP64 fallback (VB_STATUS_REFINE_STALL) and
    matches the FP64 step."""
    net = syn.make_network(41, 30, 185)
    cases, Y, K, DT, A = _batch(net, (7, 8), 24, True)
    sol, delta, st, *_ = _run(net, cases, Y, K, DT, A, max_refine=0, tol=1e-15)
    assert (st == STALL).all(), st
    dn = chem.to_device(net.tables)
    s64, d64, st64 = jstep.Ros2Step(dn, jstep.atm_from_dict(A))(Y, K, DT)
    assert (st64.cpu().numpy() == 0).all()
    s64 = s64.cpu().numpy()
    assert np.max(np.abs(sol - s64) / np.maximum(np.abs(s64), 1e-30)) <= 1e-10
