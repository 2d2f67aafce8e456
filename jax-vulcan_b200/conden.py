"""Condensation on the GPU (reference `conden.py`).

``update_conden_rates`` rewrites the condensation / evaporation rows of k;
``apply_h2o_relax_jax`` / ``apply_nh3_relax_jax`` run the implicit-Euler
cold-trap relaxation of one species (the NH3 form clamps condensation to the
layers at or below ``nh3_conden_top`` and clips the condensate), keeping the
reference names. ``CondenStatic`` holds the reference's static fields as
device tensors (batched: Dg and saturation arrays [B, ...]); the total
density n_0 and the gas mask are read from the packed atmosphere.
``CondenStatic.loop_table`` gives the ``VbCondenLoop`` table with which
``outer_loop.AdaptiveRunner(conden=...)`` runs condensation inside the loop
(``vb_loop_condense``, reference `outer_loop.py:770-800`).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .chem import as_device


class VbCondenLoop(C.Structure):
    """Mirror of ``VbCondenLoop`` in include/vulcan_b200.h."""
    _fields_ = [(n, C.c_int32) for n in ("n_re", "h2o_active", "h2o_sp", "h2o_l_s", "nh3_active", "nh3_sp",
                                         "nh3_l_s", "nh3_conden_top")] + \
               [(n, C.c_double) for n in ("start_conden_time", "h2o_m_over_rho_r2", "nh3_m_over_rho_r2")] + \
               [(n, C.c_void_p) for n in ("re_idx", "sp_idx", "coeff", "Dg_re", "sat_re", "h2o_Dg", "h2o_sat",
                                          "nh3_Dg", "nh3_sat")]


class VbRelaxParams(C.Structure):
    _fields_ = [("sp", C.c_int32), ("sp_l_s", C.c_int32), ("conden_top", C.c_int32), ("reserved", C.c_int32),
                ("m_over_rho_r2", C.c_double)]


@dataclass
class CondenStatic:
    """Reference `conden.py:20-52` fields: conden_re_idx, conden_sp_idx
    [n_re], Dg_per_re, sat_n_per_re [B, n_re, nz], coeff_per_re [n_re];
    h2o_* and nh3_* ([B, nz] arrays); the packed atmosphere ``atm_blob``
    [B, VB_ATM_DOUBLES] supplies n_0 (its M) and the gas mask."""
    conden_re_idx: object
    conden_sp_idx: object
    Dg_per_re: object
    sat_n_per_re: object
    coeff_per_re: object
    atm_blob: torch.Tensor
    h2o_active: bool = False
    h2o_idx: int = 0
    h2o_l_s_idx: int = 0
    h2o_Dg: object = None
    h2o_sat: object = None
    h2o_m_over_rho_r2: float = 0.0
    nh3_active: bool = False
    nh3_idx: int = 0
    nh3_l_s_idx: int = 0
    nh3_Dg: object = None
    nh3_sat: object = None
    nh3_m_over_rho_r2: float = 0.0
    nh3_conden_top: int = 0
    start_conden_time: float = 0.0

    def loop_table(self, batch: int, nz: int):
        """The ``VbCondenLoop`` table (device copies kept on the object)."""
        keep = self.__dict__.setdefault("_keep", {})
        re = np.asarray(self.conden_re_idx, np.int32)
        n_re = int(re.size)
        t = VbCondenLoop()
        t.n_re = n_re
        t.start_conden_time = float(self.start_conden_time)

        def dev(name, x, dtype=torch.float64, shape=None):
            a = as_device(np.asarray(x) if not torch.is_tensor(x) else x, dtype)
            if shape is not None:
                a = a.reshape(shape).contiguous()
            keep[name] = a
            return a.data_ptr() if a.numel() else None

        if n_re:
            t.re_idx = dev("re_idx", re, torch.int32)
            t.sp_idx = dev("sp_idx", np.asarray(self.conden_sp_idx, np.int32), torch.int32)
            t.coeff = dev("coeff", self.coeff_per_re)
            t.Dg_re = dev("Dg_re", self.Dg_per_re, shape=(batch, n_re, nz))
            t.sat_re = dev("sat_re", self.sat_n_per_re, shape=(batch, n_re, nz))
        if self.h2o_active:
            t.h2o_active, t.h2o_sp, t.h2o_l_s = 1, int(self.h2o_idx), int(self.h2o_l_s_idx)
            t.h2o_m_over_rho_r2 = float(self.h2o_m_over_rho_r2)
            t.h2o_Dg = dev("h2o_Dg", self.h2o_Dg, shape=(batch, nz))
            t.h2o_sat = dev("h2o_sat", self.h2o_sat, shape=(batch, nz))
        if self.nh3_active:
            t.nh3_active, t.nh3_sp, t.nh3_l_s = 1, int(self.nh3_idx), int(self.nh3_l_s_idx)
            t.nh3_conden_top = int(self.nh3_conden_top)
            t.nh3_m_over_rho_r2 = float(self.nh3_m_over_rho_r2)
            t.nh3_Dg = dev("nh3_Dg", self.nh3_Dg, shape=(batch, nz))
            t.nh3_sat = dev("nh3_sat", self.nh3_sat, shape=(batch, nz))
        return t


def update_conden_rates(k_arr, y, st: CondenStatic, stream=None):
    """Condensation rows of ``k_arr`` [B, nr+1, nz] rewritten in place
    (reference `conden.py:55-71`); returns ``k_arr``."""
    B, nz, ni = y.shape
    re = as_device(np.asarray(st.conden_re_idx, np.int32), torch.int32)
    sp = as_device(np.asarray(st.conden_sp_idx, np.int32), torch.int32)
    n_re = int(re.numel())
    Dg = as_device(st.Dg_per_re).reshape(B, n_re, nz).contiguous()
    sat = as_device(st.sat_n_per_re).reshape(B, n_re, nz).contiguous()
    coeff = as_device(st.coeff_per_re)
    # every device buffer is bound to a name until the launch is queued: a
    # temporary freed mid-call could hand its memory to the next argument
    _lib.check(_lib.lib().vb_conden_rates(B, nz, ni, k_arr.shape[1] - 1, n_re, _lib.ptr(re), _lib.ptr(sp),
                                          _lib.ptr(coeff), _lib.ptr(Dg), _lib.ptr(sat),
                                          _lib.ptr(y), _lib.ptr(k_arr), _lib.stream_handle(stream)),
               "vb_conden_rates")
    return k_arr


def _relax(y, ymix, dt, st, sp, ls, Dg, sat, m, top, stream):
    B, nz, ni = y.shape
    p = VbRelaxParams()
    p.sp, p.sp_l_s, p.conden_top, p.m_over_rho_r2 = int(sp), int(ls), int(top), float(m)
    d = as_device(np.broadcast_to(np.asarray(dt, np.float64), (B,)).copy()) if not torch.is_tensor(dt) else dt
    Dg_t = as_device(Dg).reshape(B, nz).contiguous()
    sat_t = as_device(sat).reshape(B, nz).contiguous()
    _lib.check(_lib.lib().vb_conden_relax(B, nz, ni, C.addressof(p), _lib.ptr(Dg_t), _lib.ptr(sat_t),
                                          _lib.ptr(st.atm_blob), _lib.ptr(d), _lib.ptr(y), _lib.ptr(ymix),
                                          _lib.stream_handle(stream)), "vb_conden_relax")
    return y, ymix


def apply_h2o_relax_jax(y, ymix, dt, st: CondenStatic, stream=None):
    """H2O cold trap (reference `conden.py:74-116`), in place; no-op unless
    ``h2o_active``."""
    if not st.h2o_active:
        return y, ymix
    return _relax(y, ymix, dt, st, st.h2o_idx, st.h2o_l_s_idx, st.h2o_Dg, st.h2o_sat, st.h2o_m_over_rho_r2, -1,
                  stream)


def apply_nh3_relax_jax(y, ymix, dt, st: CondenStatic, stream=None):
    """NH3 cold trap (reference `conden.py:119-160`), in place; no-op unless
    ``nh3_active``."""
    if not st.nh3_active:
        return y, ymix
    return _relax(y, ymix, dt, st, st.nh3_idx, st.nh3_l_s_idx, st.nh3_Dg, st.nh3_sat, st.nh3_m_over_rho_r2,
                  st.nh3_conden_top, stream)
