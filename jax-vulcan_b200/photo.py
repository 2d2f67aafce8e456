"""Photochemistry on the GPU (reference `photo.py`).

``compute_tau_jax``, ``compute_flux_jax``, ``compute_J_jax_flat`` and
``update_k_with_J`` keep the reference signatures; ``PhotoDevice`` holds the
cross-section tables in device memory once (the reference's ``PhotoData`` and
``PhotoJData``) and ``photo_update`` runs the in-loop photo branch
(tau -> flux -> J -> k rows, reference `outer_loop.py:283-350`).
``PhotoCarry`` holds the photo fields of the loop carry for a batch and
``photo_branch`` runs that branch for the atmospheres a device mask selects,
with the actinic-flux change the loop condition reads.
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple

import numpy as np
import torch

from . import _lib
from .chem import as_device


class VbPhoto(C.Structure):
    """Mirror of ``VbPhoto`` in include/vulcan_b200.h."""
    _fields_ = [("nbin", C.c_int32), ("n_abs", C.c_int32), ("n_abs_T", C.c_int32), ("n_scat", C.c_int32),
                ("n_br", C.c_int32), ("n_br_T", C.c_int32), ("din12", C.c_int32), ("reserved", C.c_int32),
                ("T_stride", C.c_int64), ("T_stride_J", C.c_int64),
                ("absp_idx", C.c_void_p), ("absp_T_idx", C.c_void_p), ("scat_idx", C.c_void_p),
                ("absp_cross", C.c_void_p), ("absp_T_cross", C.c_void_p), ("scat_cross", C.c_void_p),
                ("cross_J", C.c_void_p), ("cross_J_T", C.c_void_p), ("bins", C.c_void_p),
                ("sflux_top", C.c_void_p), ("br_re_idx", C.c_void_p), ("br_T_re_idx", C.c_void_p),
                ("br_active", C.c_void_p), ("br_T_active", C.c_void_p),
                ("dbin1", C.c_double), ("dbin2", C.c_double), ("mu_zenith", C.c_double), ("edd", C.c_double),
                ("ag0", C.c_double), ("hc", C.c_double), ("f_diurnal", C.c_double)]


class PhotoData(NamedTuple):
    """Absorber / scatterer tables (reference `photo.py:15-32`)."""
    absp_idx: object
    absp_cross: object
    absp_T_idx: object
    absp_T_cross: object
    scat_idx: object
    scat_cross: object


class PhotoJData(NamedTuple):
    """Branch cross sections (reference `photo.py:248-266`)."""
    cross_J: object
    cross_J_T: object
    din12_indx: int
    dbin1: float
    dbin2: float


class PhotoDevice:
    """Device copies of the photochemistry tables plus the ``VbPhoto`` struct."""

    def __init__(self, ph: dict, nz: int):
        self.keep = {}

        def dev(name, x, dtype=torch.float64):
            t = as_device(np.asarray(x), dtype)
            self.keep[name] = t
            return t

        def ptr_or_none(t):
            return t.data_ptr() if t.numel() else None

        nbin = int(np.asarray(ph["bins"]).shape[0])
        s = VbPhoto()
        s.nbin = nbin
        ai = dev("absp_idx", np.asarray(ph["absp_idx"], np.int32), torch.int32)
        ati = dev("absp_T_idx", np.asarray(ph["absp_T_idx"], np.int32), torch.int32)
        si = dev("scat_idx", np.asarray(ph["scat_idx"], np.int32), torch.int32)
        s.n_abs, s.n_abs_T, s.n_scat = ai.numel(), ati.numel(), si.numel()
        s.absp_idx, s.absp_T_idx, s.scat_idx = ptr_or_none(ai), ptr_or_none(ati), ptr_or_none(si)
        s.absp_cross = ptr_or_none(dev("absp_cross", ph["absp_cross"]))
        s.absp_T_cross = ptr_or_none(dev("absp_T_cross", ph["absp_T_cross"]))
        s.scat_cross = ptr_or_none(dev("scat_cross", ph["scat_cross"]))
        cj = dev("cross_J", ph.get("cross_J", np.zeros((0, nbin))))
        cjt = dev("cross_J_T", ph.get("cross_J_T", np.zeros((0, nz, nbin))))
        s.cross_J, s.cross_J_T = ptr_or_none(cj), ptr_or_none(cjt)
        s.n_br = cj.shape[0] if cj.dim() == 2 else 0
        s.n_br_T = cjt.shape[0] if cjt.dim() == 3 else 0
        s.bins = dev("bins", ph["bins"]).data_ptr()
        s.sflux_top = dev("sflux_top", ph["sflux_top"]).data_ptr()
        ri = dev("br_re_idx", np.asarray(ph.get("branch_re_idx", np.zeros(0)), np.int32), torch.int32)
        rti = dev("br_T_re_idx", np.asarray(ph.get("branch_T_re_idx", np.zeros(0)), np.int32), torch.int32)
        act = dev("br_active", np.asarray(ph.get("branch_active", np.ones(ri.numel(), bool)), np.uint8),
                  torch.uint8)
        actT = dev("br_T_active", np.asarray(ph.get("branch_T_active", np.ones(rti.numel(), bool)), np.uint8),
                   torch.uint8)
        s.br_re_idx, s.br_T_re_idx = ptr_or_none(ri), ptr_or_none(rti)
        s.br_active, s.br_T_active = ptr_or_none(act), ptr_or_none(actT)
        s.din12 = int(ph["din12_indx"])
        s.dbin1, s.dbin2 = float(ph["dbin1"]), float(ph["dbin2"])
        s.mu_zenith, s.edd, s.ag0 = float(ph["mu_zenith"]), float(ph["edd"]), float(ph["ag0"])
        s.hc, s.f_diurnal = float(ph["hc"]), float(ph.get("f_diurnal", 1.0))
        s.T_stride = 0
        s.T_stride_J = 0
        self.struct = s
        self.nbin = nbin
        self.nz = nz

    def with_(self, **kw):
        s = VbPhoto()
        C.memmove(C.addressof(s), C.byref(self.struct), C.sizeof(VbPhoto))
        for k, v in kw.items():
            setattr(s, k, v)
        return s


def _b(x):
    t = as_device(x)
    return (t.unsqueeze(0), True) if t.dim() == 2 else (t, False)


def compute_tau_jax(y, dz, photo: PhotoDevice, stream=None):
    """Optical depth tau[nz+1, nbin] (reference `photo.py:84-123`)."""
    yt, single = _b(y)
    B, nz, ni = yt.shape
    dzt = as_device(dz).reshape(B, nz)
    tau = torch.empty((B, nz + 1, photo.nbin), dtype=torch.float64, device=yt.device)
    _lib.check(_lib.lib().vb_photo_tau(B, nz, ni, C.addressof(photo.struct), _lib.ptr(yt), _lib.ptr(dzt),
                                       _lib.ptr(tau), _lib.stream_handle(stream)), "vb_photo_tau")
    return tau[0] if single else tau


def compute_flux_jax(tau, ymix, photo: PhotoDevice, dflux_u_prev, ag0=None, stream=None):
    """Two-stream flux -> (aflux, sflux, dflux_d, dflux_u) (reference `photo.py:126-245`).

    ``ag0`` overrides the asymmetry factor held in ``photo``."""
    tt = as_device(tau)
    single = tt.dim() == 2
    if single:
        tt = tt.unsqueeze(0)
    B, nz1, nbin = tt.shape
    nz = nz1 - 1
    ym = as_device(ymix).reshape(B, nz, -1)
    prev = as_device(dflux_u_prev).reshape(B, nz1, nbin)
    aflux = torch.empty((B, nz, nbin), dtype=torch.float64, device=tt.device)
    sflux = torch.empty_like(tt)
    dd = torch.empty_like(tt)
    du = torch.empty_like(tt)
    s = photo.struct if ag0 is None else photo.with_(ag0=float(ag0))
    _lib.check(_lib.lib().vb_photo_flux(B, nz, ym.shape[2], C.addressof(s), _lib.ptr(tt), _lib.ptr(ym),
                                        _lib.ptr(prev), _lib.ptr(aflux), _lib.ptr(sflux), _lib.ptr(dd),
                                        _lib.ptr(du), _lib.stream_handle(stream)), "vb_photo_flux")
    if single:
        return aflux[0], sflux[0], dd[0], du[0]
    return aflux, sflux, dd, du


def compute_J_jax_flat(aflux, photo: PhotoDevice, stream=None):
    """(J_br [n_br, nz], J_br_T [n_br_T, nz]) (reference `photo.py:377-392`)."""
    at = as_device(aflux)
    single = at.dim() == 2
    if single:
        at = at.unsqueeze(0)
    B, nz, nbin = at.shape
    s = photo.struct
    J = torch.empty((B, s.n_br, nz), dtype=torch.float64, device=at.device)
    JT = torch.empty((B, s.n_br_T, nz), dtype=torch.float64, device=at.device)
    _lib.check(_lib.lib().vb_photo_j(B, nz, 0, C.addressof(s), _lib.ptr(at), _lib.ptr(J) if J.numel() else None,
                                     _lib.ptr(JT) if JT.numel() else None, None, _lib.stream_handle(stream)),
               "vb_photo_j")
    return (J[0], JT[0]) if single else (J, JT)


def update_k_with_J(k_arr, aflux, photo: PhotoDevice, stream=None):
    """Write J * f_diurnal into the photolysis rows of ``k_arr`` in place for
    the active branches (reference `photo.py:455-478`), computing J from
    ``aflux`` in the same kernel. Returns ``k_arr``."""
    kt = k_arr
    single = kt.dim() == 2
    k3 = kt.unsqueeze(0) if single else kt
    at = as_device(aflux)
    at = at.unsqueeze(0) if at.dim() == 2 else at
    B, nz, nbin = at.shape
    nr = k3.shape[1] - 1
    _lib.check(_lib.lib().vb_photo_j(B, nz, nr, C.addressof(photo.struct), _lib.ptr(at), None, None, _lib.ptr(k3),
                                     _lib.stream_handle(stream)), "vb_photo_j")
    return kt


def photo_update(y, ymix, dz, k_arr, photo: PhotoDevice, dflux_u_prev, stream=None):
    """The in-loop photo branch: tau -> flux -> J -> k rows (reference
    `outer_loop.py:283-350`). Updates ``k_arr`` in place; returns
    (aflux, dflux_u)."""
    tau = compute_tau_jax(y, dz, photo, stream)
    aflux, sflux, dd, du = compute_flux_jax(tau, ymix, photo, dflux_u_prev, stream=stream)
    update_k_with_J(k_arr, aflux, photo, stream)
    return aflux, du


class PhotoCarry:
    """Photo fields of the loop carry for a batch of atmospheres (reference
    `JaxIntegState` tau, aflux, sflux, dflux_d, dflux_u, J_br, J_br_T,
    `outer_loop.py:66-80`), device tensors updated in place."""

    def __init__(self, photo: PhotoDevice, batch: int, nz: int, aflux=None, dflux_u=None):
        nbin = photo.nbin
        dev = dict(dtype=torch.float64, device="cuda")
        self.tau = torch.zeros((batch, nz + 1, nbin), **dev)
        self.aflux = (torch.zeros((batch, nz, nbin), **dev) if aflux is None
                      else as_device(aflux).reshape(batch, nz, nbin).clone())
        self.sflux = torch.zeros((batch, nz + 1, nbin), **dev)
        self.dflux_d = torch.zeros((batch, nz + 1, nbin), **dev)
        self.dflux_u = (torch.zeros((batch, nz + 1, nbin), **dev) if dflux_u is None
                        else as_device(dflux_u).reshape(batch, nz + 1, nbin).clone())
        s = photo.struct
        self.J_br = torch.zeros((batch, s.n_br, nz), **dev)
        self.J_br_T = torch.zeros((batch, s.n_br_T, nz), **dev)


def photo_branch(carry: PhotoCarry, y, ymix, dz, k_arr, photo: PhotoDevice, due=None, flux_atol=1.0, conv=None,
                 stream=None):
    """The photo branch of the adaptive loop for the atmospheres with
    ``due[b] != 0`` (all when ``due`` is None): tau -> flux -> J -> photolysis
    rows of ``k_arr`` [B, nr+1, nz] in place (reference `outer_loop.py:283-350`).
    With ``conv`` (the loop's ``VbConvState`` records), the actinic-flux
    change of each updated atmosphere is written to its record."""
    B, nz, ni = y.shape
    nr = k_arr.shape[1] - 1
    dzt = as_device(dz).reshape(-1, nz)
    if dzt.shape[0] == 1 and B > 1:
        dzt = dzt.expand(B, nz)
    dzt = dzt.contiguous()
    _lib.check(_lib.lib().vb_photo_update(
        B, nz, ni, nr, C.addressof(photo.struct), _lib.ptr(due), _lib.ptr(y), _lib.ptr(dzt), _lib.ptr(ymix),
        _lib.ptr(carry.tau), _lib.ptr(carry.aflux), _lib.ptr(carry.sflux), _lib.ptr(carry.dflux_d),
        _lib.ptr(carry.dflux_u), _lib.ptr(carry.J_br) if carry.J_br.numel() else None,
        _lib.ptr(carry.J_br_T) if carry.J_br_T.numel() else None, _lib.ptr(k_arr), float(flux_atol), _lib.ptr(conv),
        _lib.stream_handle(stream)), "vb_photo_update")
    return carry
