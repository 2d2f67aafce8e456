"""Block-tridiagonal Thomas on the GPU (reference `solver.py`).

Same call shapes as the reference: ``diag [nz, ni, ni]``, ``sup_d``/``sub_d``
``[nz-1, ni]`` (the diagonal off-diagonal blocks exactly as the reference
solver receives them), ``rhs [nz, ni]``; a leading batch axis is accepted
everywhere. The factors hold the inverses of the eliminated diagonal blocks
(reference `solver.py:23-31` keeps LU factors; both allow new right-hand
sides without refactorising).
"""
from __future__ import annotations

from typing import NamedTuple

import torch

from . import _lib
from .chem import as_device


class BlockThomasDiagFactors(NamedTuple):
    buf: torch.Tensor       # opaque device buffer (vb_bt_factor_bytes)
    batch: int
    nz: int
    ni: int
    status: torch.Tensor    # [batch] int32 status words
    single: bool


def factor_block_thomas_diag_offdiag(diag, sup_d, sub_d, stream=None) -> BlockThomasDiagFactors:
    """Factor once for reuse (reference `solver.py:33-64`)."""
    d = as_device(diag)
    single = d.dim() == 3
    if single:
        d = d.unsqueeze(0)
    B, nz, ni, _ = d.shape
    su = as_device(sup_d).reshape(B, max(nz - 1, 0), ni)
    sb = as_device(sub_d).reshape(B, max(nz - 1, 0), ni)
    L = _lib.lib()
    nbytes = int(L.vb_bt_factor_bytes(B, nz, ni))
    buf = torch.empty(nbytes, dtype=torch.uint8, device=d.device)
    status = torch.zeros(B, dtype=torch.int32, device=d.device)
    _lib.check(L.vb_bt_factor(B, nz, ni, _lib.ptr(d), _lib.ptr(su) if su.numel() else _lib.ptr(d),
                              _lib.ptr(sb) if sb.numel() else _lib.ptr(d), _lib.ptr(buf), _lib.ptr(status),
                              _lib.stream_handle(stream)), "vb_bt_factor")
    return BlockThomasDiagFactors(buf, B, nz, ni, status, single)


def _solve(factors: BlockThomasDiagFactors, rhs, transposed, stream=None):
    r = as_device(rhs).reshape(factors.batch, factors.nz, factors.ni)
    x = torch.empty_like(r)
    fn = _lib.lib().vb_bt_solve_T if transposed else _lib.lib().vb_bt_solve
    _lib.check(fn(factors.batch, factors.nz, factors.ni, _lib.ptr(factors.buf), _lib.ptr(r), _lib.ptr(x),
                  _lib.stream_handle(stream)), "vb_bt_solve")
    return x[0] if factors.single else x


def solve_block_thomas_diag_offdiag(factors: BlockThomasDiagFactors, rhs, stream=None):
    """Solve for a new right-hand side (reference `solver.py:67-112`)."""
    return _solve(factors, rhs, False, stream)


def solve_block_thomas_diag_offdiag_T(factors: BlockThomasDiagFactors, rhs, stream=None):
    """Solve the transposed system A^T x = rhs with the same factors (the
    adjoint solve of reference `steady_state_grad.py:218-219`, which factors
    ``diag^T`` with sup/sub exchanged)."""
    return _solve(factors, rhs, True, stream)


def block_thomas_diag_offdiag(diag, sup_d, sub_d, rhs, stream=None):
    """Factor + solve (reference `solver.py:115-126`)."""
    return solve_block_thomas_diag_offdiag(factor_block_thomas_diag_offdiag(diag, sup_d, sub_d, stream), rhs,
                                           stream)


class MixedFactors(NamedTuple):
    buf: torch.Tensor       # opaque device buffer (vb_bt_mixed_bytes)
    batch: int
    nz: int
    ni: int
    status: torch.Tensor    # [batch] int32 status words
    single: bool


def factor_block_thomas_mixed(diag, sup_d, sub_d, stream=None) -> MixedFactors:
    """Mixed-precision factorisation: FP32 inverses of the eliminated diagonal
    blocks (Gauss-Jordan, as the FP64 factor), the FP64 blocks kept for the
    refinement residual."""
    d = as_device(diag)
    single = d.dim() == 3
    if single:
        d = d.unsqueeze(0)
    B, nz, ni, _ = d.shape
    su = as_device(sup_d).reshape(B, max(nz - 1, 0), ni)
    sb = as_device(sub_d).reshape(B, max(nz - 1, 0), ni)
    L = _lib.lib()
    buf = torch.empty(int(L.vb_bt_mixed_bytes(B, nz, ni)), dtype=torch.uint8, device=d.device)
    status = torch.zeros(B, dtype=torch.int32, device=d.device)
    _lib.check(L.vb_bt_factor_mixed(B, nz, ni, _lib.ptr(d), _lib.ptr(su) if su.numel() else _lib.ptr(d),
                                    _lib.ptr(sb) if sb.numel() else _lib.ptr(d), _lib.ptr(buf), _lib.ptr(status),
                                    _lib.stream_handle(stream)), "vb_bt_factor_mixed")
    return MixedFactors(buf, B, nz, ni, status, single)


def solve_block_thomas_mixed(factors: MixedFactors, rhs, max_refine: int = 3, tol: float = 1e-13, stream=None):
    """Solve with FP64 iterative refinement over the FP32 factors; atmospheres
    whose refinement stalls are refactored and solved in FP64
    (VB_STATUS_REFINE_STALL in ``factors.status``). Returns (x, passes)."""
    r = as_device(rhs).reshape(factors.batch, factors.nz, factors.ni).contiguous()
    x = torch.empty_like(r)
    passes = torch.zeros(factors.batch, dtype=torch.int32, device=r.device)
    _lib.check(_lib.lib().vb_bt_solve_mixed(factors.batch, factors.nz, factors.ni, _lib.ptr(factors.buf),
                                            _lib.ptr(r), _lib.ptr(x), int(max_refine), float(tol),
                                            _lib.ptr(factors.status), _lib.ptr(passes),
                                            _lib.stream_handle(stream)), "vb_bt_solve_mixed")
    return (x[0] if factors.single else x), passes
