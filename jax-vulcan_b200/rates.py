"""Rate constants on the GPU (reference `rates.py` and `gibbs.py`).

``RateTables`` encodes a parsed network once (the forward row kinds, the
low-temperature caps, which rows get a reverse and which are removed) with
its NASA-9 coefficients in device memory; ``build_rate_array`` and
``compute_forward_k`` keep the reference signatures and run ``vb_rates``.
With ``with_dkdT`` the same launch also returns dk/dT at fixed M.
"""
from __future__ import annotations

import ctypes as C
from types import SimpleNamespace

import numpy as np
import torch

from . import _lib
from .chem import as_device
from .network import NetworkTables

VB_RK_NONE, VB_RK_ARRHENIUS, VB_RK_LINDEMANN, VB_RK_TROE_OH_CH3 = 0, 1, 2, 3
VB_RCAP = {"H + CH3 + M -> CH4 + M": 1, "H + C2H4 + M -> C2H5 + M": 2, "H + C2H5 + M -> C2H6 + M": 3}
VB_RC_THERMAL, VB_RC_REVERSE, VB_RC_DROP_FWD, VB_RC_DROP_REV = 16, 32, 64, 128
VB_RATES_LOWT_CAPS = 1
SPECIAL_OH_CH3 = "OH + CH3 + M -> CH3OH + M"


class VbRateTables(C.Structure):
    """Mirror of ``VbRateTables`` in include/vulcan_b200.h."""
    _fields_ = [("nr", C.c_int32), ("ni", C.c_int32), ("max_terms", C.c_int32), ("reserved", C.c_int32),
                ("code", C.c_void_p), ("par", C.c_void_p), ("nasa9", C.c_void_p), ("r_idx", C.c_void_p),
                ("p_idx", C.c_void_p), ("r_st", C.c_void_p), ("p_st", C.c_void_p)]


def row_codes(net: NetworkTables, remove_list=None, forward_only=False) -> np.ndarray:
    """Per forward row: the rate form (reference `rates.py:96-123`), the
    low-temperature cap (`:150-164`), whether its reverse row is filled from
    K_eq (`gibbs.py:95-103`, `:136`) and the removed rows (`rates.py:169-181`)."""
    if net.a is None:
        raise ValueError("the network tables carry no rate parameters (parse the network text)")
    code = np.zeros(net.nr + 1, dtype=np.int32)
    drop = {int(i) for i in (remove_list or ()) if 0 <= int(i) <= net.nr}
    for i in range(1, net.nr + 1, 2):
        if not net.is_forward[i]:
            continue
        runtime = net.is_photo[i] or net.is_ion[i] or net.is_conden[i] or net.is_radiative[i]
        if runtime:
            kind = VB_RK_NONE
        elif net.is_special[i]:
            if net.Rf.get(i, "").strip() == SPECIAL_OH_CH3:
                kind = VB_RK_TROE_OH_CH3
            else:
                kind = VB_RK_ARRHENIUS if net.a[i] != 0.0 else VB_RK_NONE
        elif net.has_kinf[i]:
            kind = VB_RK_LINDEMANN
        else:
            kind = VB_RK_ARRHENIUS
        c = kind | (VB_RCAP.get(net.Rf.get(i, ""), 0) << 2)
        if not forward_only:
            if i + 1 < net.stop_rev_indx:
                c |= VB_RC_REVERSE
                if not runtime:
                    c |= VB_RC_THERMAL
            if i in drop:
                c |= VB_RC_DROP_FWD
            if i + 1 in drop:
                c |= VB_RC_DROP_REV
        code[i] = c
    return code


class RateTables:
    """Device copy of a network's rate tables and NASA-9 coefficients
    [ni, 2, 10] (reference `gibbs.load_nasa9` layout)."""

    def __init__(self, net: NetworkTables, nasa9_coeffs, remove_list=None, forward_only=False):
        coeffs = np.asarray(nasa9_coeffs, np.float64)
        if coeffs.shape != (net.ni, 2, 10):
            raise ValueError(f"NASA-9 coefficients must be [{net.ni}, 2, 10], got {coeffs.shape}")
        par = np.stack([net.a, net.n, net.E, net.a_inf, net.n_inf, net.E_inf], axis=1)
        self.keep = dict(
            code=as_device(row_codes(net, remove_list, forward_only), torch.int32),
            par=as_device(par), nasa9=as_device(coeffs),
            r_idx=as_device(net.reactant_idx.astype(np.int32), torch.int32),
            p_idx=as_device(net.product_idx.astype(np.int32), torch.int32),
            r_st=as_device(net.reactant_stoich), p_st=as_device(net.product_stoich))
        s = VbRateTables()
        s.nr, s.ni, s.max_terms = net.nr, net.ni, net.reactant_idx.shape[1]
        for f in ("code", "par", "nasa9", "r_idx", "p_idx", "r_st", "p_st"):
            setattr(s, f, self.keep[f].data_ptr())
        self.struct = s
        self.nr = net.nr

    def __call__(self, T, M, lowT_caps=False, with_dkdT=False, out=None, stream=None):
        """k [B, nr+1, nz] (and dk/dT) for temperatures and densities [B, nz]
        or [nz] (then the result is [nr+1, nz])."""
        Tt = as_device(T)
        single = Tt.dim() == 1
        Tt = Tt.reshape(-1, Tt.shape[-1]).contiguous()
        Mt = as_device(M).reshape(Tt.shape).contiguous()
        B, nz = Tt.shape
        k = out if out is not None else torch.empty((B, self.nr + 1, nz), dtype=torch.float64, device=Tt.device)
        dk = torch.empty_like(k) if with_dkdT else None
        _lib.check(_lib.lib().vb_rates(B, nz, C.addressof(self.struct), _lib.ptr(Tt), _lib.ptr(Mt),
                                       VB_RATES_LOWT_CAPS if lowT_caps else 0, _lib.ptr(k), _lib.ptr(dk),
                                       _lib.stream_handle(stream)), "vb_rates")
        if single:
            k = k[0]
            dk = None if dk is None else dk[0]
        return (k, dk) if with_dkdT else k


_cache: dict = {}


def _tables(net, coeffs, remove_list, forward_only):
    key = (id(net), id(coeffs), tuple(remove_list or ()), forward_only)
    if key not in _cache:
        _cache[key] = (RateTables(net, coeffs, remove_list, forward_only), net, coeffs)
    return _cache[key][0]


def compute_forward_k(net: NetworkTables, T, M, stream=None):
    """Forward rate constants k [nr+1, nz] (reference `rates.py:61-125`):
    reverse rows and runtime-filled rows zero."""
    zeros = np.zeros((net.ni, 2, 10))
    return _tables(net, zeros, None, True)(T, M, stream=stream)


def build_rate_array(cfg, net: NetworkTables, atm, nasa9_coeffs, with_dkdT=False, stream=None):
    """Forward -> low-T caps (``cfg.use_lowT_limit_rates``) -> reverse from
    NASA-9 Gibbs -> ``cfg.remove_list`` (reference `rates.py:184-208`), for
    ``atm.Tco`` / ``atm.M`` of one atmosphere [nz] or a batch [B, nz]."""
    cfg = cfg if cfg is not None else SimpleNamespace()
    t = _tables(net, nasa9_coeffs, getattr(cfg, "remove_list", None), False)
    return t(atm.Tco, atm.M, lowT_caps=bool(getattr(cfg, "use_lowT_limit_rates", False)), with_dkdT=with_dkdT,
             stream=stream)
