"""vb_ros2_step_static (the Ros2 step whose scratch is a module-scope device
array) against vb_ros2_step (caller workspace) on the same inputs, through the
C-ABI, on two calls in a row with different shapes so that the second call
starts from the first call's scratch contents.

Tolerance: the parity bound of the step tests,
``|x - ref| <= 1e-10 * max(|sol_ref|, 1e-30)`` for sol and delta; status words
must be equal.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import load_pkg

pytestmark = pytest.mark.gpu

_lib = load_pkg("_lib")
chem = load_pkg("chem")
jstep = load_pkg("jax_step")
syn = load_pkg("synthetic")

TOL = 1e-10


def _batch(net, seed, nz, n):
    cases = [syn.make_case(seed=seed + b, net=net, nz=nz, mild=True, k_range=(-40.0, 4.0), moldiff=True)
             for b in range(n)]
    Y = np.stack([c.y for c in cases])
    K = np.stack([c.k for c in cases])
    A = {kk: (np.stack([c.atm[kk] for c in cases]) if not isinstance(cases[0].atm[kk], bool)
              else cases[0].atm[kk]) for kk in cases[0].atm}
    return Y, K, jstep.atm_from_dict(A)


def _static_step(dn, step, y, k, dt, fm):
    B, nz = y.shape[0], y.shape[1]
    sol = torch.full_like(y, float("nan"))
    delta = torch.full_like(y, float("nan"))
    status = torch.full((B,), -1, dtype=torch.int32, device="cuda")
    rc = _lib.lib().vb_ros2_step_static(
        dn.handle, B, nz, _lib.ptr(y), _lib.ptr(k), _lib.ptr(dt), _lib.ptr(step.blob), step.flags,
        _lib.ptr(fm), _lib.ptr(sol), _lib.ptr(delta), _lib.ptr(status), _lib.stream_handle())
    _lib.check(rc, "vb_ros2_step_static")
    return sol, delta, status


def test_static_scratch_step_matches_workspace_step():
    net = syn.make_network(41, 30, 185)
    dn = chem.to_device(net.tables)
    rng = np.random.default_rng(7)
    # call 1: 4 atmospheres x 24 layers; call 2: 3 x 17 with a fix mask.
    for seed, nz, n, dts, use_fm in ((60, 24, 4, [1e-6, 1e-4, 1e-8, 1e-5], False),
                                     (70, 17, 3, [1e-7, 1e-3, 1e-6], True)):
        Y, K, atm = _batch(net, seed, nz, n)
        step = jstep.Ros2Step(dn, atm, batch=n)
        y = torch.as_tensor(Y, device="cuda")
        k = torch.as_tensor(K, device="cuda")
        dt = torch.as_tensor(np.array(dts), device="cuda")
        fm = torch.as_tensor(rng.random(Y.shape) < 0.05, dtype=torch.uint8, device="cuda") if use_fm else None
        sol_ref, delta_ref, status_ref = step(y, k, dt, fix_mask=fm)
        status_ref = status_ref.clone()
        sol, delta, status = _static_step(dn, step, y, k, dt, fm)
        torch.cuda.synchronize()
        scale = torch.clamp(sol_ref.abs(), min=1e-30)
        e_sol = float(((sol - sol_ref).abs() / scale).max())
        e_del = float(((delta - delta_ref).abs() / scale).max())
        assert e_sol <= TOL, f"nz={nz}: sol err {e_sol:.3e}"
        assert e_del <= TOL, f"nz={nz}: delta err {e_del:.3e}"
        assert torch.equal(status, status_ref)


def test_static_scratch_rejects_oversize_batch():
    net = syn.make_network(41, 30, 185)
    dn = chem.to_device(net.tables)
    L = _lib.lib()
    nz = 64
    per_atm = int(L.vb_ros2_workspace_bytes(1, nz, net.tables.ni, None))
    limit = 64 << 20
    B = limit // per_atm + 1
    assert int(L.vb_ros2_workspace_bytes(B, nz, net.tables.ni, None)) > limit
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.vb_ros2_step_static(dn.handle, B, nz, dummy, dummy, dummy, dummy, 0, None, dummy, dummy,
                               dummy, None)
    assert rc == 1
    assert b"static maximum" in L.vb_last_error()
