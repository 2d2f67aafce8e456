"""Chemistry RHS and analytic Jacobian on the GPU (reference `chem.py`).

``NetworkArrays`` mirrors the reference pytree (`chem.py:28-80`): it carries
``ni``/``nr`` and the padded stoichiometry tables, here uploaded once to the
device together with the gather tables the kernels use.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .network import NetworkTables


def as_device(x, dtype=torch.float64):
    """Contiguous CUDA tensor of ``dtype`` (copies host arrays)."""
    if isinstance(x, torch.Tensor):
        t = x
        if t.device.type != "cuda":
            t = t.to("cuda")
        if t.dtype != dtype:
            t = t.to(dtype)
        return t.contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device="cuda")


class NetworkArrays:
    """Device-resident network tables (reference `chem.py:28-67`).

    ``ni`` and ``nr`` are plain ints; the tables live in device memory owned by
    the C library and are freed when this object is collected.
    """

    def __init__(self, ni, nr, reactant_idx, product_idx, reactant_stoich, product_stoich,
                 is_three_body):
        self.ni = int(ni)
        self.nr = int(nr)
        self.reactant_idx = np.ascontiguousarray(reactant_idx, dtype=np.int64)
        self.product_idx = np.ascontiguousarray(product_idx, dtype=np.int64)
        self.reactant_stoich = np.ascontiguousarray(reactant_stoich, dtype=np.float64)
        self.product_stoich = np.ascontiguousarray(product_stoich, dtype=np.float64)
        self.is_three_body = np.ascontiguousarray(is_three_body, dtype=np.uint8)
        T = self.reactant_idx.shape[1]
        if self.reactant_idx.shape != (self.nr + 1, T) or self.product_idx.shape != (self.nr + 1, T):
            raise ValueError("stoichiometry tables must be [nr+1, max_terms]")
        L = _lib.lib()
        h = C.c_void_p()
        _lib.check(L.vb_net_create(self.ni, self.nr, T,
                                   self.reactant_idx.ctypes.data, self.product_idx.ctypes.data,
                                   self.reactant_stoich.ctypes.data, self.product_stoich.ctypes.data,
                                   self.is_three_body.ctypes.data, C.byref(h)), "vb_net_create")
        self._handle = h

    @property
    def handle(self):
        return self._handle

    @property
    def max_terms(self):
        return int(self.reactant_idx.shape[1])

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().vb_net_destroy(h)
            except Exception:
                pass
            self._handle = None


def to_device(net: NetworkTables) -> NetworkArrays:
    """Pack parsed tables for the GPU (reference `chem.py:70-80` ``to_jax``)."""
    return NetworkArrays(net.ni, net.nr, net.reactant_idx, net.product_idx, net.reactant_stoich,
                         net.product_stoich, net.is_three_body)


def _batched(y, M, k):
    y = as_device(y)
    squeeze = y.dim() == 2
    if squeeze:
        y = y.unsqueeze(0)
    M = as_device(M).reshape(y.shape[0], y.shape[1])
    k = as_device(k).reshape(y.shape[0], -1, y.shape[1])
    return y, M, k, squeeze


def chem_rhs(y, M, k, net: NetworkArrays, stream=None):
    """Chemistry dy/dt, [nz, ni] or [B, nz, ni] (reference `chem.py:83-131`)."""
    y, M, k, sq = _batched(y, M, k)
    B, nz, ni = y.shape
    out = torch.empty_like(y)
    _lib.check(_lib.lib().vb_chem_rhs(net.handle, B, nz, _lib.ptr(y), _lib.ptr(M), _lib.ptr(k),
                                      _lib.ptr(out), _lib.stream_handle(stream)), "vb_chem_rhs")
    return out[0] if sq else out


def chem_jac_analytical(y, M, k, net: NetworkArrays, stream=None):
    """Analytic Jacobian, [nz, ni, ni] or [B, nz, ni, ni] (reference `chem.py:144-214`)."""
    y, M, k, sq = _batched(y, M, k)
    B, nz, ni = y.shape
    out = torch.empty((B, nz, ni, ni), dtype=torch.float64, device=y.device)
    _lib.check(_lib.lib().vb_chem_jac(net.handle, B, nz, _lib.ptr(y), _lib.ptr(M), _lib.ptr(k),
                                      _lib.ptr(out), _lib.stream_handle(stream)), "vb_chem_jac")
    return out[0] if sq else out
