"""Layer-vectorized stage 2 of the Ros2 step (a thread per layer, the rate
of every reaction and layer staged in the workspace's rate region) against
the per-layer stage-2 kernel (a CTA per layer) and the oracle.

Both sum every species list over the same terms in the reference's order
with the same operations, so the steps must agree bit for bit: sol, delta,
status and both stage vectors. Against the oracle the step's tolerance holds
(``|x - ref| <= 1e-10 max(|sol_ref|, 1e-30)``).
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
at = load_pkg("autotune")


def batch_of(cases):
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    DT = np.array([c.dt for c in cases])
    A = {key: (v if isinstance(v, bool) else np.stack([c.atm[key] for c in cases]))
         for key, v in cases[0].atm.items()}
    return Y, K, DT, A


def both_paths(dn, A, Y, K, DT, fm=None, tuning=None):
    out = []
    for assembly in (True, False):
        step = jstep.Ros2Step(dn, jstep.atm_from_dict(A), assembly=assembly)
        if tuning is not None:
            at.set_tuning(dn, tuning)
        sol, delta, status = step(Y, K, DT, fix_mask=fm)
        k1, k2 = step.stages()
        out.append([t.clone() for t in (sol, delta, status, k1, k2)])
    if tuning is not None:
        at.set_tuning(dn, {})
    return out


def assert_identical(a, b):
    for x, y, name in zip(a, b, ("sol", "delta", "status", "k1", "k2")):
        assert torch.equal(x, y), name


def test_assembly_region_size():
    net = syn.make_network(0, 69, 700)
    dn = chem.to_device(net.tables)
    L = load_pkg("_lib").lib()
    got = int(L.vb_ros2_assembly_bytes(dn.handle, 3, 120))
    assert got == 3 * 120 * (dn.nr + 1) * 8


@pytest.mark.parametrize("mild", [False, True])
def test_config0_batch_identical_and_oracle(mild):
    """Config-0 shape (ni=69, 700+700 reactions, nz=120): the specified stiff
    draw and the well-conditioned one; the oracle on the latter."""
    net = syn.make_network(0, 69, 700)
    dn = chem.to_device(net.tables)
    kw = dict(mild=True, k_range=(-40.0, 4.0)) if mild else {}
    cases = [syn.make_case(seed=(700 + b,), net=net, nz=120, **kw) for b in range(5)]
    Y, K, DT, A = batch_of(cases)
    lv, pl = both_paths(dn, A, Y, K, DT)
    assert_identical(lv, pl)
    assert int(lv[2].abs().sum()) == 0
    if mild:
        for b in (0, 4):
            sref, dref = orc.ros2_step(cases[b].y, cases[b].k, cases[b].dt, cases[b].atm, net.tables)
            scale = np.maximum(np.abs(sref), 1e-30)
            assert np.max(np.abs(lv[0][b].cpu().numpy() - sref) / scale) <= 1e-10
            assert np.max(np.abs(lv[1][b].cpu().numpy() - dref) / scale) <= 1e-10


def test_every_transport_term_fix_mask_and_three_body():
    """Molecular diffusion, advection and settling, both boundary fluxes,
    three-body reactions and a fix_mask, at a layer count that is not a
    multiple of the warp (nz=37)."""
    net = syn.make_network(61, 30, 185, n_three_body=12)
    dn = chem.to_device(net.tables)
    cases = [syn.make_case(seed=(610 + b,), net=net, nz=37, mild=True, k_range=(-40.0, 4.0), moldiff=True,
                           advection=True, fluxes=True) for b in range(3)]
    Y, K, DT, A = batch_of(cases)
    fm = np.zeros(Y.shape, dtype=np.uint8)
    fm[:, 3:9, 2] = 1
    fm[1, :, 7] = 1
    fm[2, 0, :] = 1
    lv, pl = both_paths(dn, A, Y, K, DT, fm=fm)
    assert_identical(lv, pl)
    sref, dref = orc.ros2_step(cases[1].y, cases[1].k, cases[1].dt, cases[1].atm, net.tables, fix_mask=fm[1])
    scale = np.maximum(np.abs(sref), 1e-30)
    assert np.max(np.abs(lv[0][1].cpu().numpy() - sref) / scale) <= 1e-10


def test_more_layers_than_a_tile_and_two_streams():
    """nz=150 (two layer tiles of 128) with ni=89 (the config-3 shape), and the
    two-stream step, whose halves use their own part of the region."""
    net = syn.make_network(62, 89, 1000, elements=("C", "H", "O", "N", "S"))
    dn = chem.to_device(net.tables)
    cases = [syn.make_case(seed=(620 + b,), net=net, nz=150, mild=True, k_range=(-40.0, 4.0)) for b in range(4)]
    Y, K, DT, A = batch_of(cases)
    lv, pl = both_paths(dn, A, Y, K, DT)
    assert_identical(lv, pl)
    lv2, _ = both_paths(dn, A, Y, K, DT, tuning={"streams": 2})
    assert_identical(lv2, pl)


def test_ragged_batch_identical():
    """Ragged layer counts (the zoff path), one of them above a tile."""
    net = syn.make_network(63, 30, 185)
    dn = chem.to_device(net.tables)
    nzs = [12, 140, 2, 33]
    cases = [syn.make_case(seed=(630 + b,), net=net, nz=nz, mild=True, k_range=(-40.0, 4.0), moldiff=True,
                           fluxes=True) for b, nz in enumerate(nzs)]
    dts = torch.as_tensor(np.array([1e-6, 1e-4, 1e-8, 1e-5]), device="cuda")
    res = []
    for assembly in (True, False):
        step = jstep.RaggedRos2Step(dn, [jstep.atm_from_dict(c.atm) for c in cases], assembly=assembly)
        y, k = step.pack([c.y for c in cases], [c.k for c in cases])
        sol, delta, status = step(y, k, dts)
        res.append((sol.clone(), delta.clone(), status.clone()))
    for x, y in zip(*res):
        assert torch.equal(x, y)
    assert int(res[0][2].abs().sum()) == 0


def test_mixed_step_identical():
    """The mixed-precision step (FP32 factor, FP64 refinement) with and
    without the rate region: the same stage-2 sums, so the same refinement
    passes and the same bits."""
    net = syn.make_network(0, 69, 700)
    dn = chem.to_device(net.tables)
    cases = [syn.make_case(seed=(720 + b,), net=net, nz=60, mild=True, k_range=(-40.0, 4.0)) for b in range(3)]
    Y, K, DT, A = batch_of(cases)
    res = []
    for assembly in (True, False):
        step = jstep.Ros2Step(dn, jstep.atm_from_dict(A), mixed=True, assembly=assembly)
        sol, delta, status = step(Y, K, DT)
        res.append((sol.clone(), delta.clone(), status.clone(), step.passes.clone()))
    for x, y in zip(*res):
        assert torch.equal(x, y)
