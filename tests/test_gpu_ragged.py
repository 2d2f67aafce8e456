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


def test_loop_body_and_convergence_on_a_ragged_batch():
    """vb_loop_body and vb_loop_converge with zoff: atmospheres of 12, 7 and
    10 layers packed by layers in one launch (state, rings and records at
    per-atmosphere offsets) equal the same atmospheres run alone, bit for
    bit."""
    import ctypes as C
    loop = load_pkg("outer_loop")
    _lib = load_pkg("_lib")
    L = _lib.lib()
    net = syn.make_network(51, 30, 185)
    dn = chem.to_device(net.tables)
    ni = net.tables.ni
    nzs = [12, 7, 10]
    cases = [syn.make_case(seed=(560 + b,), net=net, nz=nz, mild=True, k_range=(-40.0, 4.0), moldiff=True)
             for b, nz in enumerate(nzs)]
    dts = np.array([1e-6, 3e-6, 1e-7])
    rstep = jstep.RaggedRos2Step(dn, [jstep.atm_from_dict(c.atm) for c in cases])
    y, k = rstep.pack([c.y for c in cases], [c.k for c in cases])
    sol, delta, status = rstep(y, k, torch.as_tensor(dts, device="cuda"))
    compo = net.compo
    na = compo.shape[1]
    atom_ini = np.stack([np.einsum("zi,ia->a", c.y, compo) * (1 + 1e-7) for c in cases])
    al0 = np.stack([(np.einsum("zi,ia->a", c.y, compo) - atom_ini[b]) / atom_ini[b] for b, c in enumerate(cases)])
    ymix = [c.y / c.y.sum(axis=1, keepdims=True) for c in cases]
    Y, YP = y.clone(), y.clone()
    X = torch.as_tensor(np.concatenate(ymix), device="cuda").contiguous()
    DT = torch.as_tensor(dts, device="cuda").clone()
    AL = torch.as_tensor(al0, device="cuda").contiguous()
    ALP = AL.clone()
    rec = np.zeros(3, loop.SCALARS_DTYPE)
    rec["rtol"], rec["loss_criteria"] = 0.05, 1e-3
    SC = torch.from_numpy(rec.view(np.uint8).copy()).cuda()
    p = loop.LoopStatics().params(na)
    compo_d = torch.as_tensor(compo, device="cuda")
    ini_d = torch.as_tensor(atom_ini, device="cuda")
    sh = _lib.stream_handle()
    assert L.vb_loop_body(3, rstep.nz_max, ni, rstep.zoff.data_ptr(), C.addressof(p), rstep.blob.data_ptr(), None,
                          compo_d.data_ptr(), ini_d.data_ptr(), None, None, sol.data_ptr(), delta.data_ptr(),
                          Y.data_ptr(), YP.data_ptr(), X.data_ptr(), AL.data_ptr(), ALP.data_ptr(), DT.data_ptr(),
                          SC.data_ptr(), None, None, None, None, sh) == 0
    cs = 4
    cp = loop.ConvStatics(conv_step=cs).params()
    ring_y = torch.zeros((rstep.layers * cs, ni), dtype=torch.float64, device="cuda")
    ring_t = torch.zeros((3, cs), dtype=torch.float64, device="cuda")
    crec = np.zeros(3, loop.CONV_DTYPE)
    crec["longdy"], crec["longdydt"], crec["longdy_seen_min"] = 1.0, 1.0, np.inf
    CV = torch.from_numpy(crec.view(np.uint8).copy()).cuda()
    sm = torch.full((3,), 1e-8, dtype=torch.float64, device="cuda")
    assert L.vb_loop_converge(3, rstep.nz_max, ni, rstep.zoff.data_ptr(), C.addressof(cp), rstep.blob.data_ptr(),
                              sm.data_ptr(), None, Y.data_ptr(), X.data_ptr(), SC.data_ptr(), ring_y.data_ptr(),
                              ring_t.data_ptr(), CV.data_ptr(), None, sh) == 0
    torch.cuda.synchronize()
    z = rstep.zoff_host
    sc_all = SC.cpu().numpy().view(loop.SCALARS_DTYPE)
    cv_all = CV.cpu().numpy().view(loop.CONV_DTYPE)
    for b, c in enumerate(cases):
        step1 = jstep.Ros2Step(dn, jstep.atm_from_dict(c.atm))
        s1, d1, _ = step1(c.y, c.k, dts[b])
        st1 = loop.LoopState(c.y[None], ymix[b][None], dts[b], al0[b][None], rtol=0.05)
        loop.loop_body(st1, s1.reshape(1, *c.y.shape), d1.reshape(1, *c.y.shape), step1.blob, compo, atom_ini[b],
                       loop.LoopStatics())
        st1.enable_convergence(cs)
        loop.loop_converge(st1, step1.blob, loop.ConvStatics(conv_step=cs), 1e-8)
        torch.cuda.synchronize()
        sl = slice(int(z[b]), int(z[b + 1]))
        assert torch.equal(Y[sl], st1.y[0]) and torch.equal(YP[sl], st1.y_prev[0]) and torch.equal(X[sl], st1.ymix[0]), b
        assert torch.equal(AL[b], st1.atom_loss[0]) and torch.equal(DT[b], st1.dt[0]), b
        assert sc_all[b].tobytes() == st1.scalars_host()[0].tobytes(), b
        assert cv_all[b].tobytes() == st1.conv_host()[0].tobytes(), b
        rs = slice(int(z[b]) * cs, int(z[b + 1]) * cs)
        assert torch.equal(ring_y[rs].reshape(cs, -1, ni), st1.ring_y[0]) and torch.equal(ring_t[b], st1.ring_t[0]), b


def test_autotuned_multi_network_batch():
    """The autotuner times every candidate shape per network group on the
    device, applies the fastest (read back through vb_net_get_tuning) and the
    tuned batch still matches the oracle; a cache round trip re-applies it."""
    at = load_pkg("autotune")
    nets = [syn.make_network(54, 30, 185), syn.make_network(55, 69, 700)]
    dns = [chem.to_device(n.tables) for n in nets]
    cases, items = [], []
    for b in range(6):
        g = b % 2
        c = syn.make_case(seed=(540 + b,), net=nets[g], nz=10 + b, mild=True, k_range=(-40.0, 4.0))
        cases.append((c, 1e-6, g))
        items.append((dns[g], jstep.atm_from_dict(c.atm), c.y, c.k, 1e-6))
    batch = jstep.MultiNetworkBatch(items, tuning="tune")
    assert len(batch.tuned) == 2
    for g in batch.groups:
        key = at.group_key(g["step"].net, g["step"].batch, g["step"].layers)
        assert at.get_tuning(g["step"].net) == batch.tuned[key]["tuning"]
        assert len(batch.tuned[key]["candidates"]) == len(list(at.candidates(g["step"].net.ni)))
    batch.step()
    torch.cuda.synchronize()
    for (c, dt, g), (s, d, st) in zip(cases, batch.results()):
        sref, dref = orc.ros2_step(c.y, c.k, dt, c.atm, c.net.tables)
        check_step(s.cpu(), d.cpu(), sref, dref)
        assert int(st) == 0
    for n in dns:
        at.set_tuning(n, {})
    again = jstep.MultiNetworkBatch(items, tuning=dict(batch.tuned))
    assert len(again.tuned) == 2
    for g in again.groups:
        key = at.group_key(g["step"].net, g["step"].batch, g["step"].layers)
        assert at.get_tuning(g["step"].net) == batch.tuned[key]["tuning"]
