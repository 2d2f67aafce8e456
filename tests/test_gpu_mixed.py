"""Mixed-precision block solve (FP32 factors, FP64 iterative refinement, FP64
refactor fallback) against the FP64 oracle.

* Well-conditioned Ros2 systems (order-scaled rate constants, the shapes of
  the benchmark network): refinement converges in at most 3 passes after the
  first solve, no atmosphere falls back, and the per-species maximum relative
  error against the FP64 oracle is reported and must stay <= 1e-6 (the bound
  the mixed path is specified to); it reaches rounding level in practice.
* The SNCHO-shaped stiff systems (ni=89, nz=150, k in [1e-45, 1e-6]): FP32
  cannot resolve blocks of condition 1e25 and beyond, so refinement stalls and
  the FP64 fallback must deliver a solve whose normwise backward error stays
  at rounding level, flagged VB_STATUS_REFINE_STALL.
"""
import numpy as np
import pytest
import torch

from conftest import load_pkg
from oracle import ros2 as orc

pytestmark = pytest.mark.gpu

solver = load_pkg("solver")
syn = load_pkg("synthetic")
STALL = 4


def systems(cases):
    out = [orc.lhs_blocks(c.y, c.k, c.dt, c.atm, c.net.tables) for c in cases]
    diag = np.stack([o[0] for o in out])
    sup = np.stack([o[1] for o in out])
    sub = np.stack([o[2] for o in out])
    rhs = np.stack([o[3] for o in out])
    return diag, sup, sub, rhs


def backward_error(diag, sup, sub, rhs, x):
    res = np.einsum("zij,zj->zi", diag, x)
    res[:-1] += sup * x[1:]
    res[1:] += sub * x[:-1]
    res -= rhs
    normA = max(np.abs(diag).sum(axis=2).max(), 1.0)
    return np.abs(res).max() / (normA * np.abs(x).max() + np.abs(rhs).max())


def test_mixed_solve_converges_on_well_conditioned_systems():
    net = syn.make_network(61, 69, 700)
    cases = [syn.make_case(seed=(610 + b,), net=net, nz=40, mild=True, k_range=(-40.0, 4.0), moldiff=True)
             for b in range(4)]
    diag, sup, sub, rhs = systems(cases)
    f = solver.factor_block_thomas_mixed(diag, sup, sub)
    x, passes = solver.solve_block_thomas_mixed(f, rhs, max_refine=3, tol=1e-13)
    x = x.cpu().numpy()
    status = f.status.cpu().numpy()
    assert (status & STALL).sum() == 0, status
    assert passes.max().item() <= 4, passes
    worst = 0.0
    for b in range(len(cases)):
        ref = orc.block_thomas(diag[b], sup[b], sub[b], rhs[b])
        rel = np.abs(x[b] - ref) / np.maximum(np.abs(ref), 1e-30)
        per_species = rel.max(axis=0)
        worst = max(worst, per_species.max())
        assert per_species.max() <= 1e-6, (b, per_species.max())
    print(f"mixed solve, well conditioned: passes {passes.tolist()}, worst per-species rel err {worst:.2e}")


def test_mixed_solve_falls_back_on_stiff_systems():
    net = syn.config3_case().net
    cases = [syn.config3_case(seed=3 + b, net=net) for b in range(2)]
    diag, sup, sub, rhs = systems(cases)
    f = solver.factor_block_thomas_mixed(diag, sup, sub)
    x, passes = solver.solve_block_thomas_mixed(f, rhs, max_refine=3, tol=1e-13)
    x = x.cpu().numpy()
    status = f.status.cpu().numpy()
    for b in range(len(cases)):
        assert np.isfinite(x[b]).all()
        bwd = backward_error(diag[b], sup[b], sub[b], rhs[b], x[b])
        assert bwd < 1e-12, (b, bwd, int(status[b]), int(passes[b]))
        if status[b] & STALL:
            assert passes[b].item() == 6          # 1 + 3 FP32 passes, then 2 FP64 passes
    print(f"mixed solve, stiff: status {status.tolist()}, passes {passes.tolist()}")
