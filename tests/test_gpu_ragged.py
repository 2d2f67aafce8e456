"""Ragged and multi-network batches: atmospheres of different layer counts
(the ``zoff`` path of every kernel) and of different networks, stepped in one
batch, against the same atmospheres stepped alone and against the oracle.

Tolerances: the step's (``|x - ref| <= 1e-10 max(|sol_ref|, 1e-30)``); a
ragged batch runs each atmosphere through the same per-atmosphere arithmetic
as a batch of one, so those two must agree bit for bit.
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


def check_step(sol, delta, sol_ref, delta_ref, tol=1e-10):
    sol, delta = np.asarray(sol), np.asarray(delta)
    scale = np.maximum(np.abs(sol_ref), 1e-30)
    assert np.max(np.abs(sol - sol_ref) / scale) <= tol
    assert np.max(np.abs(delta - delta_ref) / scale) <= tol


def single(dn, c, dt):
    return jstep.jax_ros2_step(c.y, c.k, dt, jstep.atm_from_dict(c.atm), dn)


def test_ragged_one_network():
    net = syn.make_network(51, 30, 185)
    dn = chem.to_device(net.tables)
    nzs = [12, 20, 7, 2, 15]
    cases = [syn.make_case(seed=(510 + b,), net=net, nz=nz, mild=True, k_range=(-40.0, 4.0), moldiff=True,
                           fluxes=True) for b, nz in enumerate(nzs)]
    dts = np.array([1e-6, 1e-4, 1e-8, 1e-5, 1e-3])
    step = jstep.RaggedRos2Step(dn, [jstep.atm_from_dict(c.atm) for c in cases])
    y, k = step.pack([c.y for c in cases], [c.k for c in cases])
    sol, delta, status = step(y, k, torch.as_tensor(dts, device="cuda"))
    assert int(status.abs().sum()) == 0
    for b, (c, s, d) in enumerate(zip(cases, step.unpack(sol), step.unpack(delta))):
        s1, d1 = single(dn, c, dts[b])
        assert torch.equal(s, s1) and torch.equal(d, d1), b
        sref, dref = orc.ros2_step(c.y, c.k, dts[b], c.atm, c.net.tables)
        check_step(s.cpu(), d.cpu(), sref, dref)


def test_multi_network_batch_and_graph_replay():
    nets = [syn.make_network(52, 30, 185), syn.make_network(53, 69, 700)]
    dns = [chem.to_device(n.tables) for n in nets]
    rng = np.random.default_rng(5)
    cases, items = [], []
    for b in range(7):
        g = b % 2
        nz = int(rng.integers(4, 17))
        c = syn.make_case(seed=(530 + b,), net=nets[g], nz=nz, mild=True, k_range=(-40.0, 4.0))
        dt = float(10.0 ** rng.uniform(-8, -3))
        cases.append((c, dt, g))
        items.append((dns[g], jstep.atm_from_dict(c.atm), c.y, c.k, dt))
    batch = jstep.MultiNetworkBatch(items)
    batch.step()
    torch.cuda.synchronize()
    eager = [(s.clone(), d.clone()) for s, d, _ in batch.results()]
    for (c, dt, g), (s, d) in zip(cases, eager):
        s1, d1 = single(dns[g], c, dt)
        assert torch.equal(s, s1) and torch.equal(d, d1)
        sref, dref = orc.ros2_step(c.y, c.k, dt, c.atm, c.net.tables)
        check_step(s.cpu(), d.cpu(), sref, dref)
    batch.capture()
    for _ in range(2):
        batch.step()
        torch.cuda.synchronize()
        for (s, d, st), (s0, d0) in zip(batch.results(), eager):
            assert torch.equal(s, s0) and torch.equal(d, d0) and int(st) == 0
