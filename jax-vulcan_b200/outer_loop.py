"""The adaptive loop body on the GPU (reference `outer_loop.py`).

``LoopStatics`` carries the static knobs of the reference `_Statics`
(`outer_loop.py:399-490`) that the body reads; ``LoopState`` holds the
per-atmosphere carry of `JaxIntegState` (`outer_loop.py:45-135`) that the
body updates (y, y_prev, ymix, dt, t, delta, counters, atom losses, rtol,
loss_criteria) as device tensors. ``loop_body`` runs one body update after a
step; ``ConvStatics`` and ``loop_converge`` add the convergence ring, the
convergence diagnostics and the loop condition (`outer_loop.py:633-713`,
`:918-989`). ``AdaptiveRunner`` chains ``vb_ros2_step``, ``vb_loop_body``
and ``vb_loop_converge`` on one stream, so N attempts of N atmospheres run
with no host round trip (each atmosphere accepts, rejects, force-accepts and
stops on its own, as the vmapped reference runner does).
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
                ("reserved", C.c_int32), ("cond_zero_bits", C.c_uint32 * 4)] + [(n, C.c_double) for n in (
                    "loss_eps", "pos_cut", "nega_cut", "mtol", "atol", "dt_var_min", "dt_var_max", "dt_min",
                    "dt_max", "rtol_min", "rtol_max", "adapt_rtol_dec", "adapt_rtol_inc", "adapt_rtol_loss_mul",
                    "adapt_rtol_inc_loss_thresh")]


# VbLoopScalars, one record per atmosphere (72 bytes)
SCALARS_DTYPE = np.dtype([("t", "<f8"), ("delta", "<f8"), ("small_y", "<f8"), ("nega_y", "<f8"),
                          ("rtol", "<f8"), ("loss_criteria", "<f8"), ("accept_count", "<i4"),
                          ("retry_count", "<i4"), ("nega_count", "<i4"), ("loss_count", "<i4"),
                          ("delta_count", "<i4"), ("last_decision", "<i4")])
assert SCALARS_DTYPE.itemsize == 72

# VbConvState, one record per atmosphere (48 bytes)
CONV_DTYPE = np.dtype([("longdy", "<f8"), ("longdydt", "<f8"), ("longdy_seen_min", "<f8"), ("aflux_change", "<f8"),
                       ("count_since_new_min", "<i4"), ("done", "<i4"), ("update_photo_frq", "<i4"),
                       ("is_final_photo_frq", "<i4")])
assert CONV_DTYPE.itemsize == 48


class VbConvParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("conv_step", "count_min", "count_max", "conv_stall_window", "use_photo",
                                         "final_update_photo_frq", "reserved0", "reserved1")] + \
               [(n, C.c_double) for n in ("st_factor", "mtol_conv", "atol", "yconv_cri", "yconv_min", "slope_cri",
                                          "flux_cri", "trun_min", "runtime", "photo_switch_longdy",
                                          "photo_switch_longdydt")]


@dataclass
class ConvStatics:
    """Convergence and termination knobs of the reference `_Statics`
    (`outer_loop.py:420-460`), with the defaults of `vulcan_cfg.py`."""
    conv_step: int = 500
    count_min: int = 120
    count_max: int = 10000
    conv_stall_window: int = 200
    st_factor: float = 0.5
    mtol_conv: float = 1e-20
    atol: float = 0.1
    yconv_cri: float = 0.01
    yconv_min: float = 0.1
    slope_cri: float = 1e-4
    flux_cri: float = 0.1
    trun_min: float = 1e2
    runtime: float = 1e22
    use_photo: bool = False
    ini_update_photo_frq: int = 100
    final_update_photo_frq: int = 5
    photo_switch_longdy: float = 1.0      # yconv_min * 10
    photo_switch_longdydt: float = 1e-6

    def params(self) -> VbConvParams:
        p = VbConvParams()
        for n, ctype in VbConvParams._fields_:
            if hasattr(self, n):
                v = getattr(self, n)
                setattr(p, n, float(v) if ctype is C.c_double else int(v))
        return p


def slope_min_of(Kzz, Hp):
    """cond_fn's slope floor (`outer_loop.py:678-683`), per atmosphere:
    max(min(min(Kzz / (0.1 Hp[:-1])^2), 1e-8), 1e-10)."""
    Kzz, Hp = np.atleast_2d(np.asarray(Kzz)), np.atleast_2d(np.asarray(Hp))
    v = np.min(Kzz / (0.1 * Hp[:, :-1]) ** 2, axis=1)
    return np.maximum(np.minimum(v, 1e-8), 1e-10)


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
    # species indices dropped from the error norm (the reference's
    # condense_zero_mask: condense_sp + non_gas_sp when use_condense is on,
    # `outer_loop.py:244`, `:1380-1386`)
    cond_zero: tuple = ()

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
        for i in self.cond_zero:
            i = int(i)
            if not 0 <= i < 128:
                raise ValueError("cond_zero species index out of [0, 128)")
            p.cond_zero_bits[i >> 5] |= 1 << (i & 31)
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
        if self.y.dim() != 3:
            raise ValueError("y must be [B, nz, ni]")
        B = self.y.shape[0]
        self.y_prev = self.y if y_prev is None else as_device(y_prev).contiguous().clone()
        self.ymix = as_device(ymix).contiguous().clone()
        # the kernels write [B, nz, ni] arrays through these pointers: a buffer
        # of another shape would be written past its end
        for name, arr in (("y_prev", self.y_prev), ("ymix", self.ymix)):
            if tuple(arr.shape) != tuple(self.y.shape):
                raise ValueError(f"{name} must have the shape of y {tuple(self.y.shape)}, got {tuple(arr.shape)}")
        self.dt = as_device(np.broadcast_to(np.asarray(dt, np.float64), (B,)).copy())
        self.atom_loss = as_device(atom_loss).reshape(B, -1).contiguous().clone()
        self.atom_loss_prev = (self.atom_loss.clone() if atom_loss_prev is None
                               else as_device(atom_loss_prev).reshape(B, -1).contiguous().clone())
        if self.atom_loss_prev.shape != self.atom_loss.shape:
            raise ValueError("atom_loss_prev must have the shape of atom_loss")
        rec = np.zeros(B, SCALARS_DTYPE)
        rec["t"], rec["rtol"], rec["loss_criteria"] = t, rtol, loss_criteria
        rec["small_y"], rec["nega_y"] = small_y, nega_y
        for k, v in (counters or {}).items():
            rec[k] = v
        self.scalars = torch.from_numpy(rec.view(np.uint8).copy()).cuda()
        self.conv = None

    def enable_convergence(self, conv_step, longdy=1.0, longdydt=1.0, update_photo_frq=0, photo_due=False):
        """Allocates the ring buffers and the convergence carry, with the
        reference's initial values (longdy = longdydt = 1, longdy_seen_min =
        inf). ``photo_due``: whether the first attempt runs the photo branch
        (the reference's first attempt has accept_count = 0, so it does
        whenever photochemistry is on)."""
        B, nz, ni = self.y.shape
        self.conv_step = int(conv_step)
        self.ring_y = torch.zeros((B, self.conv_step, nz, ni), dtype=torch.float64, device="cuda")
        self.ring_t = torch.zeros((B, self.conv_step), dtype=torch.float64, device="cuda")
        rec = np.zeros(B, CONV_DTYPE)
        rec["longdy"], rec["longdydt"], rec["longdy_seen_min"] = longdy, longdydt, np.inf
        rec["update_photo_frq"] = update_photo_frq
        self.conv = torch.from_numpy(rec.view(np.uint8).copy()).cuda()
        self.photo_due = torch.full((B,), int(bool(photo_due)), dtype=torch.int32, device="cuda")

    def conv_host(self) -> np.ndarray:
        return self.conv.cpu().numpy().view(CONV_DTYPE)

    _FIELDS = ("y", "y_prev", "ymix", "dt", "atom_loss", "atom_loss_prev", "scalars", "conv", "ring_y", "ring_t",
               "photo_due")

    def save(self, path, stream=None, **extra):
        """Checkpoint of the carry (and of any device tensors the run owns,
        given by name: k, the packed atmosphere, the photo carry, dz) to one
        ``.npz``; ``load`` restores it bit for bit, so a run continues as if
        it had not stopped. The attempts may have been queued on another
        stream than torch's current one: ``stream`` (default: the whole
        device) is synchronised before the copies, so the checkpoint never
        holds a half-updated carry."""
        if stream is not None:
            stream.synchronize()
        else:
            torch.cuda.synchronize()
        arrays = {}
        for f in self._FIELDS:
            t = getattr(self, f, None)
            if t is not None:
                arrays["state_" + f] = t.detach().cpu().numpy()
        arrays["state_y_prev_is_y"] = np.array(self.y_prev is self.y)
        if self.conv is not None:
            arrays["state_conv_step"] = np.array(self.conv_step)
        for name, t in extra.items():
            arrays["extra_" + name] = t.detach().cpu().numpy() if torch.is_tensor(t) else np.asarray(t)
        np.savez(path, **arrays)

    @classmethod
    def load(cls, path):
        """(state, extras) from a ``save`` checkpoint: the state's tensors and
        the named extras on the current CUDA device."""
        d = np.load(path)
        st = cls.__new__(cls)
        for f in cls._FIELDS:
            key = "state_" + f
            setattr(st, f, torch.from_numpy(d[key].copy()).cuda() if key in d else None)
        if bool(d["state_y_prev_is_y"]):
            st.y_prev = st.y
        if "state_conv_step" in d:
            st.conv_step = int(d["state_conv_step"])
        extras = {k[len("extra_"):]: torch.from_numpy(d[k].copy()).cuda() for k in d.files if k.startswith("extra_")}
        return st, extras

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
              gas_mask=None, fix_mask=None, fix_y=None, zoff=None, stream=None, pre=None):
    """One body update of every atmosphere after a step (device, in place).
    ``pre`` (optional (pre_y, pre_ymix[, pre_td]) tensors) receives the
    clipped state of taken attempts (and each attempt's start time and
    step), the input of the loop's condensation and refresh."""
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
        _lib.ptr(state.dt), _lib.ptr(state.scalars), _lib.ptr(state.conv), _lib.ptr(pre[0] if pre else None),
        _lib.ptr(pre[1] if pre else None), _lib.ptr(pre[2] if pre and len(pre) > 2 else None),
        _lib.stream_handle(stream)), "vb_loop_body")


def loop_converge(state: LoopState, atm_blob, statics: ConvStatics, slope_min, ignore_mask=None, zoff=None,
                  stream=None):
    """Ring append, convergence diagnostics and the loop condition after a
    body update (device, in place; atmospheres that stop are frozen)."""
    B, nz, ni = state.y.shape
    p = statics.params()
    sm = as_device(np.broadcast_to(np.asarray(slope_min, np.float64), (B,)).copy())
    ig = None if ignore_mask is None else as_device(np.asarray(ignore_mask, np.uint8), torch.uint8)
    _lib.check(_lib.lib().vb_loop_converge(
        B, nz, ni, _lib.ptr(zoff), C.addressof(p), _lib.ptr(atm_blob), _lib.ptr(sm), _lib.ptr(ig), _lib.ptr(state.y),
        _lib.ptr(state.ymix), _lib.ptr(state.scalars), _lib.ptr(state.ring_y), _lib.ptr(state.ring_t),
        _lib.ptr(state.conv), _lib.ptr(state.photo_due), _lib.stream_handle(stream)), "vb_loop_converge")


class AdaptiveRunner:
    """Attempts of the reference loop body (`outer_loop.py:715-1100`, without
    the photo update, condensation or refresh) for a batch of atmospheres:
    each attempt is one ``vb_ros2_step`` from ``state.y`` with ``state.dt``
    followed by ``vb_loop_body`` and, given ``conv``, ``vb_loop_converge``
    (ring buffer, convergence diagnostics, loop condition); all on one
    stream. ``slope_min``: cond_fn's slope floor per atmosphere
    (``slope_min_of``).

    With ``photo`` (a ``photo.PhotoDevice``; needs ``conv`` with
    ``use_photo``), each attempt first runs the photo branch for the
    atmospheres whose photo-due flag is set (reference `outer_loop.py:716-724`:
    no retry pending and ``accept_count % update_photo_frq == 0``), which
    rewrites their photolysis rows of ``k`` in place and their actinic-flux
    change; ``dz`` [B, nz] or [nz] is the layer thickness of the photo grid
    and ``photo_carry`` (a ``photo.PhotoCarry``) the photo fields of the
    carry.

    With ``refresh`` (an ``atm_refresh.AtmRefreshStatic``), every taken
    attempt whose pre-increment accept count is a multiple of ``update_frq``
    (default 100, the reference's `update_frq`) refreshes the atmosphere from
    the attempt's clipped state (reference `outer_loop.py:813-840`): g, dzi,
    Hpi and the escape fluxes go into the
    packed atmosphere the next step reads, and ``self.dz`` (the photo grid)
    follows the refreshed layer thicknesses."""

    def __init__(self, net: NetworkArrays, atm: AtmStatic, statics: LoopStatics, compo, atom_ini,
                 batch: int | None = None, gas_mask=None, conv: ConvStatics | None = None, slope_min=1e-8,
                 ignore_mask=None, photo=None, dz=None, flux_atol=1.0, photo_carry=None, refresh=None,
                 update_frq: int = 100, conden=None):
        if photo is not None and (conv is None or not conv.use_photo):
            raise ValueError("the photo branch needs ConvStatics with use_photo")
        self.photo = photo
        self.dz = None if dz is None else as_device(dz)
        self.flux_atol = float(flux_atol)
        self.conv = conv
        self.slope_min = slope_min
        self.ignore_mask = ignore_mask
        self.step = Ros2Step(net, atm, batch)
        self.statics = statics
        self.compo = as_device(compo).contiguous()
        self.atom_ini = as_device(atom_ini)
        self.gas_mask = gas_mask
        B, nz, ni = self.step.batch, self.step.nz, net.ni
        self.sol = torch.empty((B, nz, ni), dtype=torch.float64, device="cuda")
        self.delta = torch.empty_like(self.sol)
        if photo is not None:
            from .photo import PhotoCarry
            self.photo_carry = photo_carry if photo_carry is not None else PhotoCarry(photo, B, nz)
        self.refresh = refresh
        self.update_frq = int(update_frq)
        self.conden = conden
        if refresh is not None or conden is not None:
            self.pre = (torch.empty((B, nz, ni), dtype=torch.float64, device="cuda"),
                        torch.empty((B, nz, ni), dtype=torch.float64, device="cuda"),
                        torch.empty((B, 2), dtype=torch.float64, device="cuda"))
        if conden is not None:
            self.conden_table = conden.loop_table(B, nz)
            self.gas_mask_d = None if gas_mask is None else as_device(np.asarray(gas_mask, np.uint8), torch.uint8)
        if refresh is not None:
            if update_frq < 1:
                raise ValueError("update_frq must be >= 1")
            self.mu = torch.empty((B, nz), dtype=torch.float64, device="cuda")
            self.Hp = torch.empty_like(self.mu)
            if self.dz is None:
                self.dz = torch.zeros((B, nz), dtype=torch.float64, device="cuda")
            else:
                self.dz = self.dz.reshape(-1, nz).expand(B, nz).contiguous().clone()
            self.zco = torch.empty((B, nz + 1), dtype=torch.float64, device="cuda")
            pico = as_device(refresh.pico).reshape(-1, nz + 1)
            self.pico = pico.expand(B, nz + 1).contiguous()
            self.mol_mass = as_device(refresh.mol_mass)
            self.esc = as_device(np.asarray(refresh.diff_esc_idx, np.int32), torch.int32)
            self.refresh_params = refresh.params()

    def start(self, state: LoopState):
        """Gives ``state`` its convergence carry (first attempt photo-due
        when photochemistry is on, as in the reference)."""
        c = self.conv
        state.enable_convergence(c.conv_step, update_photo_frq=c.ini_update_photo_frq if c.use_photo else 0,
                                 photo_due=c.use_photo)

    def attempt(self, state: LoopState, k, fix_mask=None, fix_y=None, stream=None):
        if self.conv is not None and state.conv is None:
            self.start(state)
        if self.photo is not None:
            from .photo import photo_branch
            if not (isinstance(k, torch.Tensor) and k.is_cuda and k.dtype == torch.float64 and k.is_contiguous()):
                raise TypeError("with the photo branch, k must be a contiguous float64 CUDA tensor (updated in place)")
            photo_branch(self.photo_carry, state.y, state.ymix, self.dz, k, self.photo, due=state.photo_due,
                         flux_atol=self.flux_atol, conv=state.conv, stream=stream)
        self.step(state.y, k, state.dt, fix_mask=fix_mask, out=(self.sol, self.delta), stream=stream)
        loop_body(state, self.sol, self.delta, self.step.blob, self.compo, self.atom_ini, self.statics,
                  gas_mask=self.gas_mask, fix_mask=fix_mask, fix_y=fix_y, stream=stream,
                  pre=self.pre if (self.refresh is not None or self.conden is not None) else None)
        if self.conden is not None:
            if not (isinstance(k, torch.Tensor) and k.is_cuda and k.dtype == torch.float64 and k.is_contiguous()):
                raise TypeError("with condensation, k must be a contiguous float64 CUDA tensor (updated in place)")
            B, nz, ni = state.y.shape
            p = self.statics.params(self.compo.shape[1])
            ini = self.atom_ini.reshape(-1, self.compo.shape[1])
            ini = (ini.expand(B, -1) if ini.shape[0] == 1 else ini).contiguous()
            _lib.check(_lib.lib().vb_loop_condense(
                B, nz, ni, k.shape[1] - 1, C.addressof(self.conden_table), C.addressof(p), _lib.ptr(self.step.blob),
                _lib.ptr(self.gas_mask_d), _lib.ptr(self.compo), _lib.ptr(ini), _lib.ptr(state.scalars),
                _lib.ptr(state.conv), _lib.ptr(self.pre[2]), _lib.ptr(self.pre[0]), _lib.ptr(self.pre[1]),
                _lib.ptr(state.y), _lib.ptr(state.y_prev), _lib.ptr(state.ymix), _lib.ptr(state.atom_loss),
                _lib.ptr(state.atom_loss_prev), _lib.ptr(k), _lib.stream_handle(stream)), "vb_loop_condense")
        if self.refresh is not None:
            B, nz, ni = state.y.shape
            _lib.check(_lib.lib().vb_loop_refresh(
                B, nz, ni, C.addressof(self.refresh_params), self.update_frq, _lib.ptr(state.scalars),
                _lib.ptr(state.conv), _lib.ptr(self.pico), _lib.ptr(self.mol_mass),
                _lib.ptr(self.esc) if self.esc.numel() else None, _lib.ptr(self.pre[0]), _lib.ptr(self.pre[1]),
                _lib.ptr(self.step.blob), _lib.ptr(self.mu), _lib.ptr(self.Hp), _lib.ptr(self.dz),
                _lib.ptr(self.zco), _lib.stream_handle(stream)), "vb_loop_refresh")
        if self.conv is not None:
            loop_converge(state, self.step.blob, self.conv, self.slope_min, self.ignore_mask, stream=stream)

    def run(self, state: LoopState, k, n_attempts: int, fix_mask=None, fix_y=None, stream=None):
        k = as_device(k).contiguous()
        for _ in range(int(n_attempts)):
            self.attempt(state, k, fix_mask, fix_y, stream)
        return state

    def run_to_convergence(self, state: LoopState, k, max_attempts: int, check_every: int = 50, fix_mask=None,
                           fix_y=None, stream=None) -> int:
        """Attempts until the loop condition stops every atmosphere
        (converged, stalled, too long or too many steps) or ``max_attempts``
        have run; the done flags are read back every ``check_every``
        attempts only, and stopped atmospheres stay frozen meanwhile.
        Returns the number of attempts run."""
        if self.conv is None:
            raise ValueError("the runner was built without ConvStatics")
        if state.conv is None:
            self.start(state)
        k = as_device(k).contiguous()
        n = 0
        while n < max_attempts:
            for _ in range(min(check_every, max_attempts - n)):
                self.attempt(state, k, fix_mask, fix_y, stream)
                n += 1
            if state.conv_host()["done"].all():
                break
        return n
