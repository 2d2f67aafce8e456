"""The adaptive loop body on the GPU (reference `outer_loop.py`).

``LoopStatics`` carries the static knobs of the reference `_Statics`
(`outer_loop.py:399-490`) that the body reads; ``LoopState`` holds the
per-atmosphere carry of `JaxIntegState` (`outer_loop.py:45-135`) that the
body updates (y, y_prev, ymix, dt, t, delta, counters, atom losses, rtol,
loss_criteria) as device tensors. ``loop_body`` runs one body update after a
step; ``AdaptiveRunner`` chains ``vb_ros2_step`` and ``vb_loop_body`` on one
stream, so N attempts of N atmospheres run with no host round trip (each
atmosphere accepts, rejects or force-accepts on its own, as the vmapped
reference runner does).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .chem import NetworkArrays, as_device
from .jax_step import AtmStatic, Ros2Step

VB_LOOP_MAX_ATOMS = 16
VB_LOOP_HYDRO_PARTIAL = 1
VB_LOOP_ZERO_BOT_ROW = 2
VB_LOOP_ADAPT_RTOL = 4


class VbLoopParams(C.Structure):
    _fields_ = [("n_atoms", C.c_int32), ("batch_max_retries", C.c_int32), ("flags", C.c_int32),
                ("adapt_rtol_dec_period", C.c_int32), ("adapt_rtol_inc_period", C.c_int32),
                ("reserved", C.c_int32)] + [(n, C.c_double) for n in (
                    "loss_eps", "pos_cut", "nega_cut", "mtol", "atol", "dt_var_min", "dt_var_max", "dt_min",
                    "dt_max", "rtol_min", "rtol_max", "adapt_rtol_dec", "adapt_rtol_inc", "adapt_rtol_loss_mul",
                    "adapt_rtol_inc_loss_thresh")]


# VbLoopScalars, one record per atmosphere (72 bytes)
SCALARS_DTYPE = np.dtype([("t", "<f8"), ("delta", "<f8"), ("small_y", "<f8"), ("nega_y", "<f8"),
                          ("rtol", "<f8"), ("loss_criteria", "<f8"), ("accept_count", "<i4"),
                          ("retry_count", "<i4"), ("nega_count", "<i4"), ("loss_count", "<i4"),
                          ("delta_count", "<i4"), ("last_decision", "<i4")])
assert SCALARS_DTYPE.itemsize == 72


@dataclass
class LoopStatics:
    """Static knobs of the body (reference `_Statics` fields of the same
    names, plus the `_make_runner` switches `non_gas_present` (given here as
    ``gas_mask``), `zero_bot_row` and `hydro_partial`)."""
    loss_eps: float = 0.1
    pos_cut: float = 0.0
    nega_cut: float = -1.0
    mtol: float = 1e-22
    atol: float = 0.1
    dt_var_min: float = 0.5
    dt_var_max: float = 2.0
    dt_min: float = 1e-14
    dt_max: float = 1e4
    batch_max_retries: int = 8
    use_adapt_rtol: bool = False
    rtol_min: float = 0.02
    rtol_max: float = 1.0
    adapt_rtol_dec_period: int = 5
    adapt_rtol_inc_period: int = 10
    adapt_rtol_dec: float = 0.5
    adapt_rtol_inc: float = 1.5
    adapt_rtol_loss_mul: float = 10.0
    adapt_rtol_inc_loss_thresh: float = 1e-3
    zero_bot_row: bool = False
    hydro_partial: bool = False

    def params(self, n_atoms: int) -> VbLoopParams:
        if not 1 <= n_atoms <= VB_LOOP_MAX_ATOMS:
            raise ValueError(f"n_atoms must be in [1, {VB_LOOP_MAX_ATOMS}]")
        p = VbLoopParams()
        p.n_atoms = n_atoms
        p.batch_max_retries = int(self.batch_max_retries)
        p.flags = ((VB_LOOP_HYDRO_PARTIAL if self.hydro_partial else 0)
                   | (VB_LOOP_ZERO_BOT_ROW if self.zero_bot_row else 0)
                   | (VB_LOOP_ADAPT_RTOL if self.use_adapt_rtol else 0))
        p.adapt_rtol_dec_period = int(self.adapt_rtol_dec_period)
        p.adapt_rtol_inc_period = int(self.adapt_rtol_inc_period)
        for n in ("loss_eps", "pos_cut", "nega_cut", "mtol", "atol", "dt_var_min", "dt_var_max", "dt_min",
                  "dt_max", "rtol_min", "rtol_max", "adapt_rtol_dec", "adapt_rtol_inc", "adapt_rtol_loss_mul",
                  "adapt_rtol_inc_loss_thresh"):
            setattr(p, n, float(getattr(self, n)))
        return p


class LoopState:
    """Per-atmosphere loop carry on the device: y, y_prev, ymix [B, nz, ni],
    atom_loss, atom_loss_prev [B, n_atoms], dt [B] and the scalar records."""

    def __init__(self, y, ymix, dt, atom_loss, atom_loss_prev=None, y_prev=None, t=0.0, rtol=0.2,
                 loss_criteria=1e-3, counters=None, small_y=0.0, nega_y=0.0):
        self.y = as_device(y).contiguous().clone()
        B = self.y.shape[0]
        self.y_prev = self.y if y_prev is None else as_device(y_prev).contiguous().clone()
        self.ymix = as_device(ymix).contiguous().clone()
        self.dt = as_device(np.broadcast_to(np.asarray(dt, np.float64), (B,)).copy())
        self.atom_loss = as_device(atom_loss).reshape(B, -1).contiguous().clone()
        self.atom_loss_prev = (self.atom_loss.clone() if atom_loss_prev is None
                               else as_device(atom_loss_prev).reshape(B, -1).contiguous().clone())
        rec = np.zeros(B, SCALARS_DTYPE)
        rec["t"], rec["rtol"], rec["loss_criteria"] = t, rtol, loss_criteria
        rec["small_y"], rec["nega_y"] = small_y, nega_y
        for k, v in (counters or {}).items():
            rec[k] = v
        self.scalars = torch.from_numpy(rec.view(np.uint8).copy()).cuda()

    @property
    def batch(self) -> int:
        return self.y.shape[0]

    def scalars_host(self) -> np.ndarray:
        return self.scalars.cpu().numpy().view(SCALARS_DTYPE)

    def snapshot(self) -> dict:
        """Host copy of the carry (field names of the reference state)."""
        rec = self.scalars_host()
        out = {k: rec[k].copy() for k in SCALARS_DTYPE.names}
        out.update(y=self.y.cpu().numpy(), y_prev=self.y_prev.cpu().numpy(), ymix=self.ymix.cpu().numpy(),
                   dt=self.dt.cpu().numpy(), atom_loss=self.atom_loss.cpu().numpy(),
                   atom_loss_prev=self.atom_loss_prev.cpu().numpy())
        return out


def loop_body(state: LoopState, sol, delta_arr, atm_blob, compo, atom_ini, statics: LoopStatics,
              gas_mask=None, fix_mask=None, fix_y=None, zoff=None, stream=None):
    """One body update of every atmosphere after a step (device, in place)."""
    B, nz, ni = state.y.shape
    compo = as_device(compo).contiguous()
    n_atoms = compo.shape[1]
    atom_ini = as_device(atom_ini).reshape(-1, n_atoms)
    if atom_ini.shape[0] == 1 and B > 1:
        atom_ini = atom_ini.expand(B, -1)
    atom_ini = atom_ini.contiguous()
    gm = None if gas_mask is None else as_device(np.asarray(gas_mask, np.uint8), torch.uint8)
    fm = None if fix_mask is None else as_device(fix_mask, torch.uint8).reshape(B, nz, ni)
    fy = None if fix_y is None else as_device(fix_y).reshape(B, nz, ni).contiguous()
    p = statics.params(n_atoms)
    _lib.check(_lib.lib().vb_loop_body(
        B, nz, ni, _lib.ptr(zoff), C.addressof(p), _lib.ptr(atm_blob), _lib.ptr(gm), _lib.ptr(compo),
        _lib.ptr(atom_ini), _lib.ptr(fm), _lib.ptr(fy), _lib.ptr(sol), _lib.ptr(delta_arr), _lib.ptr(state.y),
        _lib.ptr(state.y_prev), _lib.ptr(state.ymix), _lib.ptr(state.atom_loss), _lib.ptr(state.atom_loss_prev),
        _lib.ptr(state.dt), _lib.ptr(state.scalars), _lib.stream_handle(stream)), "vb_loop_body")


class AdaptiveRunner:
    """Attempts of the reference loop body (`outer_loop.py:715-1100`, without
    photo, condensation, refresh or the convergence ring) for a batch of
    atmospheres: each attempt is one ``vb_ros2_step`` from ``state.y`` with
    ``state.dt`` followed by ``vb_loop_body``; both stay on one stream."""

    def __init__(self, net: NetworkArrays, atm: AtmStatic, statics: LoopStatics, compo, atom_ini,
                 batch: int | None = None, gas_mask=None):
        self.step = Ros2Step(net, atm, batch)
        self.statics = statics
        self.compo = as_device(compo).contiguous()
        self.atom_ini = as_device(atom_ini)
        self.gas_mask = gas_mask
        B, nz, ni = self.step.batch, self.step.nz, net.ni
        self.sol = torch.empty((B, nz, ni), dtype=torch.float64, device="cuda")
        self.delta = torch.empty_like(self.sol)

    def attempt(self, state: LoopState, k, fix_mask=None, fix_y=None, stream=None):
        self.step(state.y, k, state.dt, fix_mask=fix_mask, out=(self.sol, self.delta), stream=stream)
        loop_body(state, self.sol, self.delta, self.step.blob, self.compo, self.atom_ini, self.statics,
                  gas_mask=self.gas_mask, fix_mask=fix_mask, fix_y=fix_y, stream=stream)

    def run(self, state: LoopState, k, n_attempts: int, fix_mask=None, fix_y=None, stream=None):
        k = as_device(k).contiguous()
        for _ in range(int(n_attempts)):
            self.attempt(state, k, fix_mask, fix_y, stream)
        return state
