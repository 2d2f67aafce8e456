"""The Ros2 step on the GPU (reference `jax_step.py`).

``jax_ros2_step(y, k_arr, dt, atm, net, fix_mask=None) -> (sol, delta_arr)``
keeps the reference signature and semantics (`jax_step.py:249-315`): y and
the outputs are ``[nz, ni]`` (or ``[B, nz, ni]`` for a batch, the reference's
vmap), ``k_arr`` is ``[nr+1, nz]``, ``dt`` a scalar (or ``[B]``), ``atm`` an
``AtmStatic``. Everything runs in the CUDA kernels of ``libvulcan_b200.so``;
``Ros2Step`` keeps the packed atmosphere, workspace and status buffers across
calls for loops that step the same atmospheres repeatedly.
"""
from __future__ import annotations

from typing import NamedTuple

import numpy as np
import torch

from . import _lib
from .chem import NetworkArrays, as_device


class AtmStatic(NamedTuple):
    """Atmosphere held constant within a step (reference `jax_step.py:26-49`).

    Arrays may be NumPy or torch; with a leading batch axis all atmospheres
    of a batch share the four flags.
    """
    Kzz: object        # (nz-1,)
    Dzz: object        # (nz-1, ni)
    dzi: object        # (nz-1,)
    vz: object         # (nz-1,)
    Hpi: object        # (nz-1,)
    Ti: object         # (nz-1,)
    Tco: object        # (nz,)
    g: object          # (nz,)
    ms: object         # (ni,)
    alpha: object      # (ni,)
    M: object          # (nz,)
    vm: object         # (nz, ni)
    vs: object         # (nz-1, ni)
    top_flux: object   # (ni,)
    bot_flux: object   # (ni,)
    bot_vdep: object   # (ni,)
    gas_indx_mask: object  # (ni,) bool
    use_vm_mol: bool
    use_settling: bool
    use_topflux: bool
    use_botflux: bool


def atm_from_dict(d) -> AtmStatic:
    return AtmStatic(**{k: d[k] for k in AtmStatic._fields})


def atm_flags(atm: AtmStatic) -> int:
    return ((_lib.VB_USE_VM_MOL if bool(atm.use_vm_mol) else 0)
            | (_lib.VB_USE_SETTLING if bool(atm.use_settling) else 0)
            | (_lib.VB_USE_TOPFLUX if bool(atm.use_topflux) else 0)
            | (_lib.VB_USE_BOTFLUX if bool(atm.use_botflux) else 0))


def pack_atm(atm: AtmStatic) -> torch.Tensor:
    """Pack an AtmStatic (optionally batched) into the device blob layout of
    ``VB_ATM_DOUBLES`` (include/vulcan_b200.h). Returns ``[B, doubles]``."""
    Tco = as_device(atm.Tco)
    batched = Tco.dim() == 2
    Tco = Tco if batched else Tco.unsqueeze(0)
    B, nz = Tco.shape

    def f(x, shape):
        t = as_device(x)
        return t.reshape((B,) + shape) if batched else t.reshape((1,) + shape)

    ms = f(atm.ms, (-1,))
    ni = ms.shape[1]

    def pad_z(t):                                  # [B, nz-1, ...] -> [B, nz, ...]
        z = torch.zeros((B, 1) + tuple(t.shape[2:]), dtype=t.dtype, device=t.device)
        return torch.cat([t, z], dim=1)

    parts = [
        pad_z(f(atm.Kzz, (nz - 1,))), pad_z(f(atm.dzi, (nz - 1,))), pad_z(f(atm.vz, (nz - 1,))),
        pad_z(f(atm.Hpi, (nz - 1,))), pad_z(f(atm.Ti, (nz - 1,))), Tco, f(atm.g, (nz,)), f(atm.M, (nz,)),
        pad_z(f(atm.Dzz, (nz - 1, ni))), f(atm.vm, (nz, ni)), pad_z(f(atm.vs, (nz - 1, ni))),
        ms, f(atm.alpha, (ni,)), f(atm.top_flux, (ni,)), f(atm.bot_flux, (ni,)), f(atm.bot_vdep, (ni,)),
        f(np.asarray(atm.gas_indx_mask, dtype=np.float64) if not isinstance(atm.gas_indx_mask, torch.Tensor)
          else atm.gas_indx_mask.to(torch.float64), (ni,)),
    ]
    blob = torch.cat([p.reshape(B, -1) for p in parts], dim=1).contiguous()
    assert blob.shape[1] == nz * (8 + 3 * ni) + 6 * ni
    return blob


class Ros2Step:
    """Reusable batched Ros2 step for ``batch`` atmospheres of one network.

    Holds the packed atmosphere, the solver workspace and the status words,
    so repeated calls allocate nothing.
    """

    def __init__(self, net: NetworkArrays, atm: AtmStatic, batch: int | None = None, mixed: bool = False,
                 max_refine: int = 3, tol: float = 1e-12, assembly: bool = True):
        """``mixed=True``: the mixed-precision step (``vb_ros2_step_mixed``:
        FP32 row-equilibrated factor on the TF32 tensor cores, FP64 refinement
        of both stages, at most ``max_refine`` passes to ``tol``, FP64
        fallback); ``self.passes`` then holds the passes run per atmosphere.
        ``assembly``: allocate the rate region of the layer-vectorized
        stage 2 (``vb_ros2_assembly_bytes``: nr+1 doubles per layer), so the
        stage-2 right-hand side is formed with a thread per layer; False: the
        per-layer stage-2 kernel (same results, less memory)."""
        self.net = net
        self.mixed = bool(mixed)
        self.max_refine = int(max_refine)
        self.tol = float(tol)
        self.blob = pack_atm(atm)
        self.flags = atm_flags(atm)
        self.batch = self.blob.shape[0] if batch is None else int(batch)
        if self.blob.shape[0] != self.batch:
            if self.blob.shape[0] != 1:
                raise ValueError("atm batch does not match")
            self.blob = self.blob.expand(self.batch, -1).contiguous()
        ni = net.ni
        self.nz = (self.blob.shape[1] - 6 * ni) // (8 + 3 * ni)
        L = _lib.lib()
        size = L.vb_ros2_mixed_workspace_bytes if self.mixed else L.vb_ros2_workspace_bytes
        self.ws_bytes = int(size(self.batch, self.nz, ni, None))
        if assembly:
            self.ws_bytes = ((self.ws_bytes + 255) & ~255) + int(
                L.vb_ros2_assembly_bytes(net.handle, self.batch, self.nz))
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device="cuda")
        self.status = torch.zeros(self.batch, dtype=torch.int32, device="cuda")
        self.passes = torch.zeros(self.batch, dtype=torch.int32, device="cuda")

    def __call__(self, y, k, dt, fix_mask=None, out=None, stream=None):
        """Returns (sol, delta, status) as device tensors of the batch shape."""
        B, nz, ni = self.batch, self.nz, self.net.ni
        y = as_device(y).reshape(B, nz, ni)
        k = as_device(k).reshape(B, self.net.nr + 1, nz)
        dt = as_device(dt).reshape(-1)
        if dt.numel() == 1 and B > 1:
            dt = dt.expand(B).contiguous()
        fm = None if fix_mask is None else as_device(fix_mask, torch.uint8).reshape(B, nz, ni)
        if out is None:
            sol = torch.empty_like(y)
            delta = torch.empty_like(y)
        else:
            sol, delta = out
        if self.mixed:
            _lib.check(_lib.lib().vb_ros2_step_mixed(
                self.net.handle, B, nz, None, _lib.ptr(y), _lib.ptr(k), _lib.ptr(dt), _lib.ptr(self.blob),
                self.flags, _lib.ptr(fm), self.max_refine, self.tol, _lib.ptr(sol), _lib.ptr(delta),
                _lib.ptr(self.status), _lib.ptr(self.passes), _lib.ptr(self.ws), self.ws_bytes,
                _lib.stream_handle(stream)), "vb_ros2_step_mixed")
        else:
            _lib.check(_lib.lib().vb_ros2_step(
                self.net.handle, B, nz, None, _lib.ptr(y), _lib.ptr(k), _lib.ptr(dt), _lib.ptr(self.blob),
                self.flags, _lib.ptr(fm), _lib.ptr(sol), _lib.ptr(delta), _lib.ptr(self.status),
                _lib.ptr(self.ws), self.ws_bytes, _lib.stream_handle(stream)), "vb_ros2_step")
        return sol, delta, self.status

    def stages(self, stream=None):
        """(k1, k2) of the last call, ``[B, nz, ni]``: the two block solves of
        the step (reference `jax_step.py:300-311`), read back from the
        workspace (``vb_ros2_stages``)."""
        B, nz, ni = self.batch, self.nz, self.net.ni
        k1 = torch.empty((B, nz, ni), dtype=torch.float64, device="cuda")
        k2 = torch.empty_like(k1)
        _lib.check(_lib.lib().vb_ros2_stages(self.net.handle, B, nz, None, _lib.ptr(self.ws), _lib.ptr(k1),
                                             _lib.ptr(k2), _lib.stream_handle(stream)), "vb_ros2_stages")
        return k1, k2


def set_wait_limit(polls: int | None) -> None:
    """Poll limit of the first bounded wait on each bulk copy in the factor
    and sweep kernels (``vb_set_wait_limit``); ``None`` restores the default.
    For failure-detection tests: a wait that runs out gives the atmosphere
    ``VB_STATUS_WATCHDOG`` and the kernel returns early."""
    _lib.check(_lib.lib().vb_set_wait_limit(-1 if polls is None else int(polls)), "vb_set_wait_limit")


def set_pipeline_wait_limit(polls: int | None) -> None:
    """Poll limit of the waits between the warps of the pipelined factor
    (``vb_set_pipeline_wait_limit``); ``None`` restores the default. For
    failure-detection tests: a wait that runs out ends every wait of the
    atmosphere's factor and gives it ``VB_STATUS_WATCHDOG``."""
    _lib.check(_lib.lib().vb_set_pipeline_wait_limit(-1 if polls is None else int(polls)),
               "vb_set_pipeline_wait_limit")


class RaggedRos2Step:
    """Ros2 step for atmospheres of one network with different layer counts
    (the ``zoff`` path of ``vb_ros2_step``).

    State, rates and the atmosphere are packed by layers: atmosphere b holds
    layers ``zoff[b]..zoff[b+1]-1`` of ``y [L, ni]``, the block
    ``[nr+1, nz_b]`` at ``k[zoff[b]*(nr+1):]`` and its own atmosphere blob.
    ``pack`` / ``unpack`` convert from and to per-atmosphere arrays.
    """

    def __init__(self, net: NetworkArrays, atms, assembly: bool = True):
        """``assembly``: allocate the rate region of the layer-vectorized
        stage 2 (as ``Ros2Step``; sized for ``batch`` atmospheres of the
        largest layer count)."""
        self.net = net
        atms = list(atms)
        self.batch = len(atms)
        blobs = [pack_atm(a)[0] for a in atms]
        flags = {atm_flags(a) for a in atms}
        if len(flags) != 1:
            raise ValueError("all atmospheres of a ragged batch share the four transport flags")
        self.flags = flags.pop()
        ni = net.ni
        self.nzs = [int((b.numel() - 6 * ni) // (8 + 3 * ni)) for b in blobs]
        if min(self.nzs) < 2:
            raise ValueError("every atmosphere needs nz >= 2")
        self.nz_max = max(self.nzs)
        self.zoff_host = np.concatenate([[0], np.cumsum(self.nzs)]).astype(np.int64)
        self.zoff = torch.as_tensor(self.zoff_host, device="cuda")
        self.layers = int(self.zoff_host[-1])
        self.blob = torch.cat(blobs).contiguous()
        L = _lib.lib()
        self.ws_bytes = int(L.vb_ros2_workspace_bytes(self.batch, self.nz_max, ni, self.zoff_host.ctypes.data))
        if assembly:
            self.ws_bytes = ((int(L.vb_ros2_workspace_bytes(self.batch, self.nz_max, ni, None)) + 255) & ~255) + \
                int(L.vb_ros2_assembly_bytes(net.handle, self.batch, self.nz_max))
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device="cuda")
        self.status = torch.zeros(self.batch, dtype=torch.int32, device="cuda")

    def pack(self, ys, ks):
        """Per-atmosphere y [nz_b, ni] and k [nr+1, nz_b] -> packed device tensors."""
        y = torch.cat([as_device(v).reshape(-1, self.net.ni) for v in ys]).contiguous()
        k = torch.cat([as_device(v).reshape(-1) for v in ks]).contiguous()
        return y, k

    def unpack(self, t):
        """Packed [L, ni] -> list of [nz_b, ni] views."""
        return [t[self.zoff_host[b]:self.zoff_host[b + 1]] for b in range(self.batch)]

    def __call__(self, y, k, dt, fix_mask=None, out=None, stream=None):
        """y [L, ni], k [sum (nr+1)*nz_b], dt [B] -> (sol, delta, status)."""
        y = as_device(y).reshape(self.layers, self.net.ni)
        k = as_device(k).reshape(-1)
        if k.numel() != self.layers * (self.net.nr + 1):
            raise ValueError("k must hold (nr+1)*nz_b values per atmosphere")
        dt = as_device(dt).reshape(-1)
        if dt.numel() == 1 and self.batch > 1:
            dt = dt.expand(self.batch).contiguous()
        fm = None if fix_mask is None else as_device(fix_mask, torch.uint8).reshape(self.layers, self.net.ni)
        if out is None:
            sol = torch.empty_like(y)
            delta = torch.empty_like(y)
        else:
            sol, delta = out
        _lib.check(_lib.lib().vb_ros2_step(
            self.net.handle, self.batch, self.nz_max, _lib.ptr(self.zoff), _lib.ptr(y), _lib.ptr(k), _lib.ptr(dt),
            _lib.ptr(self.blob), self.flags, _lib.ptr(fm), _lib.ptr(sol), _lib.ptr(delta), _lib.ptr(self.status),
            _lib.ptr(self.ws), self.ws_bytes, _lib.stream_handle(stream)), "vb_ros2_step")
        return sol, delta, self.status


class MultiNetworkBatch:
    """One Ros2 step for atmospheres of several networks and uneven layer
    counts (the batched use of the reference step under ``vmap``, one group
    per network): the groups run on their own CUDA streams, and ``capture``
    records the whole batch step as one CUDA graph for replay.

    ``cases``: sequence of ``(net, atm, y, k, dt)`` with ``y [nz, ni]``,
    ``k [nr+1, nz]``; results come back in the order given. ``tuning``:
    launch shapes per group from the autotuner (``autotune.py``): a cache
    dict, the path of a cache file, or "tune" to time the candidates now
    (``self.tuned`` records what was applied).
    """

    def __init__(self, cases, tuning=None):
        cases = list(cases)
        groups = {}
        for idx, (net, atm, y, k, dt) in enumerate(cases):
            groups.setdefault(id(net), []).append(idx)
        self.groups = []
        for idxs in groups.values():
            net = cases[idxs[0]][0]
            step = RaggedRos2Step(net, [cases[i][1] for i in idxs])
            y, k = step.pack([cases[i][2] for i in idxs], [cases[i][3] for i in idxs])
            dt = torch.as_tensor(np.array([float(cases[i][4]) for i in idxs]), dtype=torch.float64, device="cuda")
            sol, delta = torch.empty_like(y), torch.empty_like(y)
            self.groups.append(dict(idx=idxs, step=step, y=y, k=k, dt=dt, sol=sol, delta=delta,
                                    stream=torch.cuda.Stream()))
        self.batch = len(cases)
        self.graph = None
        self.tuned = {}
        if tuning is not None:
            from . import autotune
            if isinstance(tuning, str) and tuning == "tune":
                self.tuned = autotune.tune_batch(self)
            else:
                cache = autotune.load_cache(tuning) if isinstance(tuning, str) else dict(tuning)
                autotune.apply_cache(self, cache)
                self.tuned = {k: v for k, v in cache.items()
                              if k in {autotune.group_key(g["step"].net, g["step"].batch, g["step"].layers)
                                       for g in self.groups}}

    def _launch(self):
        main = torch.cuda.current_stream()
        for g in self.groups:
            g["stream"].wait_stream(main)
            with torch.cuda.stream(g["stream"]):
                g["step"](g["y"], g["k"], g["dt"], out=(g["sol"], g["delta"]), stream=g["stream"])
        for g in self.groups:
            main.wait_stream(g["stream"])

    def step(self):
        """Steps every atmosphere (replays the graph when captured)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch()

    def capture(self):
        """Records one batch step (all groups) as a CUDA graph."""
        self._launch()                     # warm: kernel attributes set outside capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch()
        self.graph = g
        return g

    def results(self):
        """(sol, delta, status) per atmosphere, in the order of ``cases``."""
        out = [None] * self.batch
        for g in self.groups:
            sols, deltas = g["step"].unpack(g["sol"]), g["step"].unpack(g["delta"])
            for j, i in enumerate(g["idx"]):
                out[i] = (sols[j], deltas[j], g["step"].status[j])
        return out


def jax_ros2_step(y, k_arr, dt, atm: AtmStatic, net: NetworkArrays, fix_mask=None):
    """One 2nd-order Rosenbrock step -> (sol, delta_arr) (reference `jax_step.py:249-315`).

    Accepts a single atmosphere (``y [nz, ni]``) or a batch (``y [B, nz, ni]``,
    ``k_arr [B, nr+1, nz]``, ``dt`` scalar or ``[B]``, batched ``atm``).
    """
    yt = as_device(y)
    single = yt.dim() == 2
    B = 1 if single else yt.shape[0]
    step = Ros2Step(net, atm, batch=B)
    sol, delta, _ = step(yt, k_arr, dt, fix_mask=fix_mask)
    if single:
        return sol[0], delta[0]
    return sol, delta


def diffusion(y, atm: AtmStatic, stream=None):
    """Eddy + molecular diffusion of a state (reference `jax_step.py:67-246`).

    Returns (diff [.., nz, ni] with boundary fluxes, diag_d [.., nz, ni] with the
    deposition term, sup_d [.., nz-1, ni], sub_d [.., nz-1, ni]) where
    ``diag_d``/``sup_d``/``sub_d`` are ``A_eddy+A_mol`` (+ bot_vdep term),
    ``B[:-1]`` and ``C[1:]`` of `jax_step.py:275-283`.
    """
    yt = as_device(y)
    single = yt.dim() == 2
    if single:
        yt = yt.unsqueeze(0)
    B, nz, ni = yt.shape
    blob = pack_atm(atm)
    if blob.shape[0] != B:
        blob = blob.expand(B, -1).contiguous()
    diff = torch.empty_like(yt)
    diag_d = torch.empty_like(yt)
    sup = torch.empty((B, nz - 1, ni), dtype=torch.float64, device=yt.device)
    sub = torch.empty_like(sup)
    _lib.check(_lib.lib().vb_diffusion(B, nz, ni, _lib.ptr(yt), _lib.ptr(blob), atm_flags(atm),
                                       _lib.ptr(diff), _lib.ptr(diag_d), _lib.ptr(sup), _lib.ptr(sub),
                                       _lib.stream_handle(stream)), "vb_diffusion")
    if single:
        return diff[0], diag_d[0], sup[0], sub[0]
    return diff, diag_d, sup, sub
