"""Implicit-function-theorem gradients of the converged state (reference
`steady_state_grad.py`), computed with the GPU kernels.

At a steady state f(y*, theta) = 0, so dL/dtheta = -(J_y^{-T} dL/dy*) . df/dtheta.
``implicit_cotangents`` assembles J_y, solves the transposed block-tridiagonal
system with the block-Thomas factors and applies the VJP kernels to every
leaf of the reference `SteadyStateInputs`. ``temperature_cotangent`` adds the
path through the rate constants (dk/dT from ``rates``) to the temperature
leaves.

``DifferentiableSteadyState`` is the ``torch.autograd.Function`` counterpart of
the reference's ``differentiable_steady_state`` custom_vjp (`:284-330`):
identity in the forward pass, the implicit k-gradient in the backward pass.
"""
from __future__ import annotations

import torch

from . import _lib
from .chem import NetworkArrays, as_device
from .jax_step import AtmStatic, atm_flags, pack_atm


def _batch(y, k):
    yt = as_device(y)
    single = yt.dim() == 2
    if single:
        yt = yt.unsqueeze(0)
    B, nz, ni = yt.shape
    kt = as_device(k).reshape(B, -1, nz)
    return yt, kt, single


def residual(y, k_arr, atm: AtmStatic, net: NetworkArrays, stream=None):
    """f(y) = chem_rhs(y) + diffusion(y) (reference `steady_state_grad.py:116-130`)."""
    yt, kt, single = _batch(y, k_arr)
    B, nz, ni = yt.shape
    blob = pack_atm(atm)
    if blob.shape[0] != B:
        blob = blob.expand(B, -1).contiguous()
    f = torch.empty_like(yt)
    _lib.check(_lib.lib().vb_residual(net.handle, B, nz, None, _lib.ptr(yt), _lib.ptr(kt), _lib.ptr(blob),
                                      atm_flags(atm), _lib.ptr(f), _lib.stream_handle(stream)), "vb_residual")
    return f[0] if single else f


def validate_steady_state_solution(y_star, k_arr, atm, net, residual_rtol=1e-6, residual_atol=0.0):
    """Residual gate before implicit AD (reference `steady_state_grad.py:178-196`)."""
    r = residual(y_star, k_arr, atm, net)
    resid_inf = float(r.abs().max())
    scale = float(as_device(y_star).abs().max())
    tol = max(residual_atol, residual_rtol * max(scale, 1.0))
    if resid_inf > tol:
        raise ValueError(
            "Steady-state residual is too large for reliable implicit differentiation: "
            f"||f||_inf={resid_inf:.3e} exceeds tolerance {tol:.3e}.")
    return resid_inf


def unpack_atm_cotangents(g_atm, nz, ni):
    """Blob of cotangents ([B][VB_ATM_DOUBLES]) -> the reference leaf arrays
    (interface arrays [B][nz-1], layer arrays [B][nz], per-species [B][ni])."""
    B = g_atm.shape[0]
    o, out = 0, {}
    for name in ("Kzz", "dzi", "vz", "Hpi", "Ti", "Tco", "g", "M"):
        out[name] = g_atm[:, o:o + nz]
        o += nz
    for name in ("Dzz", "vm", "vs"):
        out[name] = g_atm[:, o:o + nz * ni].reshape(B, nz, ni)
        o += nz * ni
    for name in ("ms", "alpha", "top_flux", "bot_flux", "bot_vdep"):
        out[name] = g_atm[:, o:o + ni]
        o += ni
    for name in ("Kzz", "dzi", "vz", "Hpi", "Ti", "Dzz", "vs"):   # interface arrays: nz-1 used
        out[name] = out[name][:, :nz - 1]
    del out["M"]          # the chemistry's M cotangent comes from vb_adjoint
    out["Kzz_transport"] = out.pop("Kzz")   # the same cotangent as vb_adjoint's Kzz, by differentiation
    return out


def implicit_cotangents(y_star, k_arr, atm: AtmStatic, net: NetworkArrays, v, stream=None):
    """Cotangents -lambda . df/dtheta with lambda = J_y^{-T} v (reference `_ssi_bwd`,
    `steady_state_grad.py:214-230`) for every leaf of the reference
    `SteadyStateInputs` (`steady_state_grad.py:36-59`): a dict with ``lambda``,
    ``k_arr``, ``M``, ``Kzz``, ``Dzz``, ``dzi``, ``vz``, ``Hpi``, ``Ti``, ``Tco``,
    ``g``, ``ms``, ``alpha``, ``vm``, ``vs``, ``top_flux``, ``bot_flux``,
    ``bot_vdep`` and ``status``."""
    yt, kt, single = _batch(y_star, k_arr)
    B, nz, ni = yt.shape
    vt = as_device(v).reshape(B, nz, ni)
    blob = pack_atm(atm)
    if blob.shape[0] != B:
        blob = blob.expand(B, -1).contiguous()
    L = _lib.lib()
    ws_bytes = int(L.vb_ros2_workspace_bytes(B, nz, ni, None))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=yt.device)
    dev = yt.device
    out = dict(
        **{"lambda": torch.empty_like(yt)},
        k_arr=torch.empty_like(kt), M=torch.empty((B, nz), dtype=torch.float64, device=dev),
        Kzz=torch.empty((B, nz - 1), dtype=torch.float64, device=dev),
        top_flux=torch.empty((B, ni), dtype=torch.float64, device=dev),
        bot_flux=torch.empty((B, ni), dtype=torch.float64, device=dev),
        bot_vdep=torch.empty((B, ni), dtype=torch.float64, device=dev),
        status=torch.zeros(B, dtype=torch.int32, device=dev))
    # Kzz cotangents are packed by layers (nz slots per atmosphere)
    kzz_full = torch.empty((B, nz), dtype=torch.float64, device=dev)
    _lib.check(L.vb_adjoint(net.handle, B, nz, None, _lib.ptr(yt), _lib.ptr(kt), _lib.ptr(blob), atm_flags(atm),
                            _lib.ptr(vt), _lib.ptr(out["lambda"]), _lib.ptr(out["k_arr"]), _lib.ptr(out["M"]),
                            _lib.ptr(kzz_full), _lib.ptr(out["top_flux"]), _lib.ptr(out["bot_flux"]),
                            _lib.ptr(out["bot_vdep"]), _lib.ptr(out["status"]), _lib.ptr(ws), ws_bytes,
                            _lib.stream_handle(stream)), "vb_adjoint")
    out["Kzz"] = kzz_full[:, :nz - 1]
    # every other transport leaf, from the blob of cotangents (vb_adjoint_atm)
    g_atm = torch.empty_like(blob)
    _lib.check(L.vb_adjoint_atm(B, nz, ni, None, _lib.ptr(yt), _lib.ptr(blob), atm_flags(atm), _lib.ptr(out["lambda"]),
                                _lib.ptr(g_atm), _lib.stream_handle(stream)), "vb_adjoint_atm")
    out.update(unpack_atm_cotangents(g_atm, nz, ni))
    if single:
        out = {kk: (vv[0] if kk != "status" else vv) for kk, vv in out.items()}
    return out


def temperature_cotangent(cot, dkdT=None):
    """dL/dT per layer [B, nz] (or [nz]) at fixed M: the Tco leaf, the
    interface temperatures Ti = (T_j + T_{j+1}) / 2 (reference
    `atm_setup.py:371`) and, given ``dkdT`` [B, nr+1, nz] from
    ``rates.build_rate_array(..., with_dkdT=True)``, the rate constants:
    g_T[j] = g_Tco[j] + (g_Ti[j-1] + g_Ti[j]) / 2 + sum_r g_k[r, j] dk_r/dT[j]."""
    gT = cot["Tco"].clone()
    gTi = cot["Ti"]
    gT[..., :-1] += 0.5 * gTi
    gT[..., 1:] += 0.5 * gTi
    if dkdT is not None:
        gT += (cot["k_arr"] * dkdT.reshape(cot["k_arr"].shape)).sum(dim=-2)
    return gT


class DifferentiableSteadyState(torch.autograd.Function):
    """y* as a differentiable function of k_arr (reference `differentiable_steady_state`,
    `steady_state_grad.py:284-330`): forward is the identity on y*; backward
    returns -(df/dk)^T J_y^{-T} (dL/dy*)."""

    @staticmethod
    def forward(ctx, k_arr, y_star, atm, net):
        ctx.save_for_backward(k_arr, y_star)
        ctx.atm = atm
        ctx.net = net
        return y_star.clone()

    @staticmethod
    def backward(ctx, grad_y):
        k_arr, y_star = ctx.saved_tensors
        cot = implicit_cotangents(y_star, k_arr, ctx.atm, ctx.net, grad_y)
        return cot["k_arr"].reshape(k_arr.shape), None, None, None


def differentiable_steady_state(k_arr, y_star, atm, net):
    return DifferentiableSteadyState.apply(k_arr, y_star, atm, net)


def steady_state_value_and_grad(loss_fn, k_arr, y_star, atm, net, residual_rtol=1e-6, residual_atol=0.0):
    """Loss of the steady state and its implicit gradients (reference
    `steady_state_grad.py:254-281`). ``loss_fn`` maps a torch y* to a scalar;
    returns (loss, cotangent dict)."""
    validate_steady_state_solution(y_star, k_arr, atm, net, residual_rtol, residual_atol)
    y = as_device(y_star).clone().requires_grad_(True)
    loss = loss_fn(y)
    (v,) = torch.autograd.grad(loss, [y])
    return loss.detach(), implicit_cotangents(y_star, k_arr, atm, net, v)
