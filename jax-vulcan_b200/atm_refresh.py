"""Atmosphere refresh on the GPU (reference `atm_refresh.py`).

``AtmRefreshStatic`` carries the reference's static fields; ``refresh`` runs
``vb_atm_refresh`` on a batch: the hydrostatic integration (mu, g, Hp, dz,
zco, dzi, Hpi) and the diffusion-limited escape fluxes in one launch, with
g, dzi, Hpi and the escape entries of top_flux written into the packed
atmosphere the Ros2 step reads (the splice of reference
`outer_loop.py:729-730`). ``update_mu_dz_jax`` keeps the reference name and
return tuple for one atmosphere.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .chem import as_device


class VbRefreshParams(C.Structure):
    _fields_ = [("pref_indx", C.c_int32), ("n_esc", C.c_int32)] + \
               [(n, C.c_double) for n in ("zco_pref", "gs", "Rp", "kb", "Navo", "max_flux")]


@dataclass
class AtmRefreshStatic:
    """Static inputs of the refresh (reference `atm_refresh.py:17-33`):
    pico [nz+1] or [B, nz+1], mol_mass [ni], diff_esc_idx, pref_indx,
    zco_pref, gs, Rp, kb, Navo, max_flux. Tco, ms and Dzz come from the
    packed atmosphere."""
    pico: object
    mol_mass: object
    diff_esc_idx: object
    pref_indx: int
    zco_pref: float
    gs: float
    Rp: float
    kb: float = 1.38064852e-16
    Navo: float = 6.02214086e23
    max_flux: float = 1e13

    def params(self) -> VbRefreshParams:
        p = VbRefreshParams()
        p.pref_indx, p.n_esc = int(self.pref_indx), int(np.asarray(self.diff_esc_idx).size)
        for n in ("zco_pref", "gs", "Rp", "kb", "Navo", "max_flux"):
            setattr(p, n, float(getattr(self, n)))
        return p


def refresh(y, ymix, atm_blob, st: AtmRefreshStatic, stream=None):
    """Refresh a batch in place in ``atm_blob`` [B, VB_ATM_DOUBLES]; returns
    (mu, Hp, dz, zco) device tensors."""
    B, nz, ni = y.shape
    dev = y.device
    pico = as_device(st.pico).reshape(-1, nz + 1)
    if pico.shape[0] == 1 and B > 1:
        pico = pico.expand(B, -1)
    pico = pico.contiguous()
    esc = as_device(np.asarray(st.diff_esc_idx, np.int32), torch.int32)
    mm = as_device(st.mol_mass)
    mu = torch.empty((B, nz), dtype=torch.float64, device=dev)
    Hp, dz = torch.empty_like(mu), torch.empty_like(mu)
    zco = torch.empty((B, nz + 1), dtype=torch.float64, device=dev)
    p = st.params()
    _lib.check(_lib.lib().vb_atm_refresh(B, nz, ni, C.addressof(p), _lib.ptr(pico), _lib.ptr(mm),
                                         _lib.ptr(esc) if esc.numel() else None, _lib.ptr(y), _lib.ptr(ymix),
                                         _lib.ptr(atm_blob), _lib.ptr(mu), _lib.ptr(Hp), _lib.ptr(dz), _lib.ptr(zco),
                                         _lib.stream_handle(stream)), "vb_atm_refresh")
    return mu, Hp, dz, zco


def blob_fields(atm_blob, nz, ni):
    """Views of the refreshed fields of the packed atmosphere: g [B, nz],
    dzi, Hpi [B, nz-1], top_flux [B, ni] (field order of the C header)."""
    return dict(g=atm_blob[:, 6 * nz:7 * nz], dzi=atm_blob[:, nz:2 * nz - 1], Hpi=atm_blob[:, 3 * nz:4 * nz - 1],
                top_flux=atm_blob[:, 8 * nz + 3 * nz * ni + 2 * ni:8 * nz + 3 * nz * ni + 3 * ni])


def update_mu_dz_jax(ymix, atm_blob, st: AtmRefreshStatic, y=None, stream=None):
    """(mu, g, Hp, dz, zco, dzi, Hpi) of one atmosphere [nz, ni] (reference
    `atm_refresh.py:36-100`); the escape fluxes of the same launch land in the
    blob's top_flux."""
    x = as_device(ymix)
    nz, ni = x.shape
    yy = as_device(y if y is not None else ymix).reshape(1, nz, ni).contiguous()
    blob = atm_blob.reshape(1, -1)
    mu, Hp, dz, zco = refresh(yy, x.reshape(1, nz, ni).contiguous(), blob, st, stream)
    f = blob_fields(blob, nz, ni)
    return mu[0], f["g"][0], Hp[0], dz[0], zco[0], f["dzi"][0], f["Hpi"][0]
