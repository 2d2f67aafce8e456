"""The rate-constant build on the GPU (``vb_rates``) against the reference's
own rates.py / gibbs.py output (``tests/golden/rates.npz``) and the oracle.

Tolerances: forward rows 1e-14 relative (CUDA's exp / log / pow are within a
few ulp of the host libm; the products and sums round as the reference's;
measured 4.9e-16); reverse rows 1e-12 relative: K_eq = exp(sum st g)
amplifies the absolute error of the g/RT sums by the size of the exponent
(measured 1.4e-14); dk/dT 1e-11 relative to max(|dk/dT|, 1e-12 |k| / T)
(measured 1.1e-13).
"""
import ctypes as C
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from conftest import golden, load_pkg
from oracle import rates as orr

pytestmark = pytest.mark.gpu

rates = load_pkg("rates")
network = load_pkg("network")


def case():
    g = golden("rates.npz")
    return g, network.parse_network_text(str(g["net_text"]))


def rel_rows(got, ref, rows):
    got, ref = np.asarray(got)[rows], ref[rows]
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300), initial=0.0))


def test_rates_match_reference():
    g, net = case()
    fwd, rev = np.arange(1, net.nr + 1, 2), np.arange(2, net.nr + 1, 2)
    cfg = SimpleNamespace(use_lowT_limit_rates=True, remove_list=list(g["remove"]))
    k = rates.build_rate_array(cfg, net, SimpleNamespace(Tco=g["T"], M=g["M"]), g["coeffs"]).cpu().numpy()
    ef, er = rel_rows(k, g["k_all"], fwd), rel_rows(k, g["k_all"], rev)
    print(f"rates vs reference: forward {ef:.2e}, reverse {er:.2e}")
    assert ef <= 1e-14 and er <= 1e-12
    assert np.array_equal(k[0], np.zeros_like(k[0]))
    assert np.array_equal(k == 0, g["k_all"] == 0)
    k2 = rates.build_rate_array(None, net, SimpleNamespace(Tco=g["T"], M=g["M"]), g["coeffs"]).cpu().numpy()
    assert rel_rows(k2, g["k_nocap"], fwd) <= 1e-14 and rel_rows(k2, g["k_nocap"], rev) <= 1e-12
    kf = rates.compute_forward_k(net, g["T"], g["M"]).cpu().numpy()
    assert rel_rows(kf, g["k_fwd"], np.arange(net.nr + 1)) <= 1e-14


def test_rates_temperature_derivative():
    """dk/dT at fixed M by dual numbers against the oracle's complex step,
    and the value part of the dual launch equal to the plain launch."""
    g, net = case()
    cfg = SimpleNamespace(use_lowT_limit_rates=True, remove_list=list(g["remove"]))
    atm = SimpleNamespace(Tco=g["T"], M=g["M"])
    k, dk = rates.build_rate_array(cfg, net, atm, g["coeffs"], with_dkdT=True)
    k0 = rates.build_rate_array(cfg, net, atm, g["coeffs"])
    assert torch.equal(k, k0)
    ref = orr.dk_dT(net, g["coeffs"], g["T"], g["M"], lowT_caps=True, remove_list=list(g["remove"]))
    kr = g["k_all"]
    scale = np.maximum(np.abs(ref), 1e-12 * np.abs(kr) / g["T"][None, :] + 1e-300)
    err = float(np.max(np.abs(dk.cpu().numpy() - ref) / scale))
    print(f"dk/dT vs complex step: {err:.2e}")
    assert err <= 1e-11


def test_rates_batch_with_per_atmosphere_temperatures():
    """Four atmospheres with temperature offsets in one launch: each equals
    its single-atmosphere launch bit for bit and the oracle within the bounds
    above."""
    g, net = case()
    T = np.stack([g["T"] + 37.0 * b for b in range(4)])
    M = np.stack([g["M"] * (1.0 + 0.1 * b) for b in range(4)])
    t = rates.RateTables(net, g["coeffs"], remove_list=list(g["remove"]))
    k = t(T, M, lowT_caps=True).cpu().numpy()
    fwd, rev = np.arange(1, net.nr + 1, 2), np.arange(2, net.nr + 1, 2)
    for b in range(4):
        assert np.array_equal(k[b], t(T[b], M[b], lowT_caps=True).cpu().numpy())
        ref = orr.build_rate_array(net, g["coeffs"], T[b], M[b], lowT_caps=True, remove_list=list(g["remove"]))
        assert rel_rows(k[b], ref, fwd) <= 1e-14 and rel_rows(k[b], ref, rev) <= 1e-12, b


def test_rates_reject_bad_arguments():
    L = load_pkg("_lib").lib()
    g, net = case()
    t = rates.RateTables(net, g["coeffs"])
    s = rates.VbRateTables()
    C.memmove(C.addressof(s), C.addressof(t.struct), C.sizeof(s))
    s.nr = 3
    dummy = C.c_void_p(16)  # never dereferenced: argument checks come first
    assert L.vb_rates(1, 4, C.addressof(s), dummy, dummy, 0, dummy, None, None) == 1
    assert b"nr even" in L.vb_last_error()
    assert L.vb_rates(1, 4, C.addressof(t.struct), None, dummy, 0, dummy, None, None) == 1
    torch.cuda.synchronize()
