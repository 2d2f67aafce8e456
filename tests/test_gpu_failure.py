"""Failure detection of the step in the forms allowed on a shared GPU: the
failures are made on the host (non-finite inputs) or by a bounded wait that is
told to give up at once; nothing faults, traps or hangs a GPU.

* NaN in one atmosphere's state and +inf in another's rate constants give
  those atmospheres VB_STATUS_NONFINITE; the other atmospheres of the batch
  keep status 0 and their results bit for bit.
* ``vb_set_wait_limit(0)``: the first bounded wait on every bulk copy of the
  factor and sweep kernels gives up, each atmosphere gets VB_STATUS_WATCHDOG
  and the kernels return after draining their copies; with the default limit
  restored the next step is correct again.
* ``vb_set_pipeline_wait_limit(0)`` with the pipelined factor: the first wait
  of a warp for a step another warp publishes gives up, that warp stops every
  other warp's wait, each atmosphere gets VB_STATUS_WATCHDOG; with the limit
  restored the next step equals the first bit for bit.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg

pytestmark = pytest.mark.gpu

_lib = load_pkg("_lib")
chem = load_pkg("chem")
jstep = load_pkg("jax_step")
syn = load_pkg("synthetic")

NONFINITE, WATCHDOG = 2, 8


def _batch(n=4, nz=20):
    net = syn.make_network(41, 30, 185)
    cases = [syn.make_case(seed=500 + b, net=net, nz=nz, mild=True, k_range=(-40.0, 4.0)) for b in range(n)]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    dn = chem.to_device(net.tables)
    return dn, jstep.Ros2Step(dn, jstep.atm_from_dict(A)), Y, K, np.full(n, 1e-6)


def _step(step, Y, K, DT):
    y = torch.as_tensor(Y, device="cuda")
    k = torch.as_tensor(K, device="cuda")
    dt = torch.as_tensor(DT, device="cuda")
    sol, delta, status = step(y, k, dt)
    torch.cuda.synchronize()
    return sol.cpu().numpy(), delta.cpu().numpy(), status.cpu().numpy().copy()


def test_nonfinite_inputs_flag_only_their_atmospheres():
    dn, step, Y, K, DT = _batch()
    sol0, delta0, st0 = _step(step, Y, K, DT)
    assert (st0 == 0).all()
    Y1, K1 = Y.copy(), K.copy()
    Y1[1, 7, 3] = np.nan                      # a NaN mixing ratio in atmosphere 1
    row = int(np.flatnonzero(K1[2, :, 5] > 0)[0])
    K1[2, row, 5] = np.inf                    # an infinite rate constant in atmosphere 2
    sol, delta, st = _step(step, Y1, K1, DT)
    assert st[1] & NONFINITE and st[2] & NONFINITE, st
    assert st[0] == 0 and st[3] == 0, st
    for b in (0, 3):
        assert np.array_equal(sol[b], sol0[b]) and np.array_equal(delta[b], delta0[b])
    assert not np.isfinite(sol[1]).all() and not np.isfinite(sol[2]).all()


def test_wait_limit_gives_watchdog_status_and_recovers():
    dn, step, Y, K, DT = _batch()
    sol0, delta0, st0 = _step(step, Y, K, DT)
    assert (st0 == 0).all()
    try:
        jstep.set_wait_limit(0)
        _, _, st = _step(step, Y, K, DT)
    finally:
        jstep.set_wait_limit(None)
    assert (st & WATCHDOG).all(), st
    sol, delta, st2 = _step(step, Y, K, DT)
    assert (st2 == 0).all(), st2
    assert np.array_equal(sol, sol0) and np.array_equal(delta, delta0)


def test_pipeline_wait_limit_gives_watchdog_status_and_recovers():
    dn, step, Y, K, DT = _batch()
    try:
        _lib.check(_lib.lib().vb_set_factor_kernel(2), "vb_set_factor_kernel")
        sol0, delta0, st0 = _step(step, Y, K, DT)
        assert (st0 == 0).all()
        try:
            jstep.set_pipeline_wait_limit(0)
            _, _, st = _step(step, Y, K, DT)
        finally:
            jstep.set_pipeline_wait_limit(None)
        assert (st & WATCHDOG).all(), st
        sol, delta, st2 = _step(step, Y, K, DT)
    finally:
        _lib.check(_lib.lib().vb_set_factor_kernel(1), "vb_set_factor_kernel")
    assert (st2 == 0).all(), st2
    assert np.array_equal(sol, sol0) and np.array_equal(delta, delta0)


def test_paired_factor_wait_limit_gives_watchdog_status_and_recovers():
    """The two-atmospheres-per-CTA factor (69 species, an odd batch: one pair
    and the last atmosphere by the single kernel) reports VB_STATUS_WATCHDOG
    for every atmosphere when its bulk-copy waits give up at once, and the
    next step equals the first bit for bit."""
    net = syn.make_network(169, 69, 700)
    cases = [syn.make_case(seed=800 + b, net=net, nz=12, mild=True, k_range=(-40.0, 4.0)) for b in range(3)]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    step = jstep.Ros2Step(chem.to_device(net.tables), jstep.atm_from_dict(A))
    DT = np.full(3, 1e-6)
    try:
        _lib.check(_lib.lib().vb_set_factor_kernel(3), "vb_set_factor_kernel")
        sol0, delta0, st0 = _step(step, Y, K, DT)
        assert (st0 == 0).all()
        try:
            jstep.set_wait_limit(0)
            _, _, st = _step(step, Y, K, DT)
        finally:
            jstep.set_wait_limit(None)
        assert (st & WATCHDOG).all(), st
        sol, delta, st2 = _step(step, Y, K, DT)
    finally:
        _lib.check(_lib.lib().vb_set_factor_kernel(1), "vb_set_factor_kernel")
    assert (st2 == 0).all(), st2
    assert np.array_equal(sol, sol0) and np.array_equal(delta, delta0)
