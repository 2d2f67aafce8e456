"""The FP64 block-factor kernels (``vb_set_factor_kernel``): 0 = blocked
Gauss-Jordan with the rank-8 trailing updates on the FP64 tensor cores, 1 =
scalar Gauss-Jordan (default), 2 = the scalar elimination pipelined per column
panel (mbarrier-signalled steps, no block barrier per step; the same
arithmetic as 1, so its results equal 1's bit for bit). Each is checked on the
Ros2 step against the
oracle (well-conditioned draws, the step bound 1e-10 relative), on the
reference's block-Thomas systems (1e-10), on the transposed solve the adjoint
uses, and on the stiff config-0 draw by the normwise backward error of both
stage solves. That bound is 1e-11 here: both kernels solve with explicit
block inverses, whose backward error on these blocks (Schur block condition
numbers ~1e29) reaches 1.4e-12 on seed 10 for either kernel (the reference's
LU substitution stays near 1e-26); the seeds of the timed batch stay below
1e-12 (tests/test_gpu_bench_inputs.py)."""
import numpy as np
import pytest
import torch

from conftest import golden, load_pkg
from oracle import ros2 as orc

pytestmark = pytest.mark.gpu

_lib = load_pkg("_lib")
chem = load_pkg("chem")
jstep = load_pkg("jax_step")
solver = load_pkg("solver")
syn = load_pkg("synthetic")


@pytest.fixture(params=[0, 1, 2, 3], ids=["blocked_dmma", "scalar_gj", "pipelined_gj", "paired_gj"])
def variant(request):
    _lib.check(_lib.lib().vb_set_factor_kernel(request.param), "vb_set_factor_kernel")
    yield request.param
    _lib.check(_lib.lib().vb_set_factor_kernel(1), "vb_set_factor_kernel")


def rel(a, b, floor=1e-30):
    return float(np.max(np.abs(np.asarray(a) - b) / np.maximum(np.abs(b), floor)))


@pytest.mark.parametrize("ni,n_fwd,nz", [(12, 30, 10), (30, 185, 40), (69, 700, 120), (89, 1000, 60)])
def test_step_matches_oracle(variant, ni, n_fwd, nz):
    elements = ("C", "H", "O", "N", "S") if ni == 89 else ("C", "H", "O", "N")
    net = syn.make_network(70 + ni, ni, n_fwd, elements)
    case = syn.make_case(seed=71, net=net, nz=nz, mild=True, k_range=(-40.0, 4.0), moldiff=True)
    sref, dref = orc.ros2_step(case.y, case.k, case.dt, case.atm, net.tables)
    dn = chem.to_device(net.tables)
    sol, delta = jstep.jax_ros2_step(case.y, case.k, case.dt, jstep.atm_from_dict(case.atm), dn)
    assert rel(sol.cpu().numpy(), sref) <= 1e-10
    assert float(np.max(np.abs(delta.cpu().numpy() - dref) / np.maximum(np.abs(sref), 1e-30))) <= 1e-10


def test_reference_block_thomas_systems(variant):
    g = golden("thomas.npz")
    x = solver.block_thomas_diag_offdiag(g["diag_small_diag"], g["diag_small_sup"], g["diag_small_sub"],
                                         g["diag_small_rhs"]).cpu().numpy()
    assert rel(x, g["diag_small_x"], 1e-12) <= 1e-10
    rng = np.random.default_rng(7)
    rng.standard_normal((8, 5, 5)); rng.standard_normal((7, 5)); rng.standard_normal((7, 5))
    rng.standard_normal((8, 5))
    d2 = rng.standard_normal((120, 93, 93)) + 1e10 * np.eye(93)
    su2 = rng.standard_normal((119, 93)) * 1e-3
    sb2 = rng.standard_normal((119, 93)) * 1e-3
    r2 = rng.standard_normal((120, 93))
    x2 = solver.block_thomas_diag_offdiag(d2, su2, sb2, r2).cpu().numpy()
    assert rel(x2, g["diag_big_x"], 1e-12) <= 1e-10


def test_transposed_solve(variant):
    rng = np.random.default_rng(5)
    nz, ni = 20, 69
    diag = rng.standard_normal((nz, ni, ni))
    diag = diag + (5.0 + np.abs(diag).sum(axis=2))[:, :, None] * np.eye(ni)[None]
    su = 0.1 * rng.standard_normal((nz - 1, ni))
    sb = 0.1 * rng.standard_normal((nz - 1, ni))
    rhs = rng.standard_normal((nz, ni))
    f = solver.factor_block_thomas_diag_offdiag(diag, su, sb)
    xT = solver.solve_block_thomas_diag_offdiag_T(f, rhs).cpu().numpy()
    assert rel(xT, orc.block_thomas(np.transpose(diag, (0, 2, 1)), sb, su, rhs), 1e-12) <= 1e-10


def test_stiff_draw_stage_backward_errors(variant):
    net = syn.make_network(0, 69, 700)
    cases = [syn.make_case(seed=(s,), net=net) for s in (0, 5, 10)]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    dn = chem.to_device(net.tables)
    step = jstep.Ros2Step(dn, jstep.atm_from_dict(A))
    sol, delta, status = step(Y, K, np.array([c.dt for c in cases]))
    k1, k2 = step.stages()
    assert (status.cpu().numpy() == 0).all()
    k1, k2 = k1.cpu().numpy(), k2.cpu().numpy()
    for b, c in enumerate(cases):
        bwd = orc.stage_backward_errors(c.y, c.k, c.dt, c.atm, net.tables, k1[b], k2[b])
        assert max(bwd) < 1e-11, (b, bwd)


@pytest.mark.parametrize("ni,n_fwd", [(12, 30), (30, 185), (69, 700), (89, 1000)])
def test_pipelined_equals_scalar_bit_for_bit(ni, n_fwd):
    """The pipelined elimination performs the scalar kernel's operations in
    the same order on the same values (only the hand-over between warps
    differs), on a ragged batch (layer counts 2..20; partial last panels and
    warps without columns at ni=12 and 30) of one network."""
    elements = ("C", "H", "O", "N", "S") if ni == 89 else ("C", "H", "O", "N")
    net = syn.make_network(90 + ni, ni, n_fwd, elements)
    dn = chem.to_device(net.tables)
    nzs = [12, 20, 7, 3, 2, 15]
    cases = [syn.make_case(seed=(600 + b,), net=net, nz=nz, mild=True, k_range=(-40.0, 4.0), moldiff=True)
             for b, nz in enumerate(nzs)]
    dts = torch.as_tensor(np.array([1e-6, 1e-4, 1e-8, 1e-5, 1e-3, 1e-7]), device="cuda")
    step = jstep.RaggedRos2Step(dn, [jstep.atm_from_dict(c.atm) for c in cases])
    y, k = step.pack([c.y for c in cases], [c.k for c in cases])
    out = {}
    try:
        for v in (1, 2):
            _lib.check(_lib.lib().vb_set_factor_kernel(v), "vb_set_factor_kernel")
            sol, delta, status = step(y, k, dts)
            torch.cuda.synchronize()
            out[v] = (sol.clone(), delta.clone(), status.clone())
    finally:
        _lib.check(_lib.lib().vb_set_factor_kernel(1), "vb_set_factor_kernel")
    assert int(out[2][2].abs().sum()) == 0
    assert torch.equal(out[1][0], out[2][0]) and torch.equal(out[1][1], out[2][1])


@pytest.mark.parametrize("batch", [4, 5])
def test_paired_equals_scalar_bit_for_bit(batch):
    """Two atmospheres per CTA with their pivot chains interleaved perform
    each atmosphere's operations in the scalar kernel's order, so the step
    equals the scalar kernel's bit for bit (an odd batch: the last
    atmosphere by the single kernel)."""
    net = syn.make_network(169, 69, 700)
    dn = chem.to_device(net.tables)
    cases = [syn.make_case(seed=(700 + b,), net=net, nz=24, mild=True, k_range=(-40.0, 4.0), moldiff=True)
             for b in range(batch)]
    Y = torch.as_tensor(np.stack([c.y for c in cases]), device="cuda")
    K = torch.as_tensor(np.stack([c.k for c in cases]), device="cuda")
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool) else cases[0].atm[kk])
         for kk in cases[0].atm}
    dt = torch.as_tensor(np.array([1e-6, 1e-4, 1e-8, 1e-5, 1e-3][:batch]), device="cuda")
    step = jstep.Ros2Step(dn, jstep.atm_from_dict(A), batch=batch)
    out = {}
    try:
        for v in (1, 3):
            _lib.check(_lib.lib().vb_set_factor_kernel(v), "vb_set_factor_kernel")
            sol, delta, status = step(Y, K, dt)
            torch.cuda.synchronize()
            out[v] = (sol.clone(), delta.clone(), status.clone())
    finally:
        _lib.check(_lib.lib().vb_set_factor_kernel(1), "vb_set_factor_kernel")
    assert int(out[3][2].abs().sum()) == 0
    assert torch.equal(out[1][0], out[3][0]) and torch.equal(out[1][1], out[3][1])
    sref, dref = orc.ros2_step(cases[0].y, cases[0].k, 1e-6, cases[0].atm, net.tables)
    assert rel(out[3][0][0].cpu().numpy(), sref) <= 1e-10
