"""Photochemistry kernels against the reference-generated fixture and the oracle.

Tolerance: 1e-12 relative for tau, the direct beam and J (floor 1e-300);
1e-11 for the diffuse fluxes and the actinic flux, relative to the largest
value of the same bin. exp() and the reduction order over absorbers and bins
differ from the reference by a few ulp; the two-stream recursions accumulate
them over the nz layers (1/chi amplifies each step slightly).
"""
import numpy as np
import pytest
import torch

from conftest import golden, load_pkg
from oracle import photo as op

pytestmark = pytest.mark.gpu
photo = load_pkg("photo")
syn = load_pkg("synthetic")


def rel(a, b, floor=1e-300):
    a = np.asarray(a)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor), initial=0.0))


def rel_bin(a, b):
    a = np.asarray(a)
    scale = np.maximum(np.max(np.abs(b), axis=0, keepdims=True), 1e-300)
    return float(np.max(np.abs(a - b) / scale, initial=0.0))


def _ph(g):
    return {k[3:]: (g[k].item() if g[k].ndim == 0 else g[k]) for k in g if k.startswith("ph_")}


def test_photo_against_reference_fixture():
    g = golden("photo.npz")
    ph = _ph(g)
    nz = g["y"].shape[0]
    dev = photo.PhotoDevice(ph, nz)
    tau = photo.compute_tau_jax(g["y"], g["dz"], dev).cpu().numpy()
    assert rel(tau, g["tau"]) <= 1e-12
    for tag, ag0 in (("ag0", 0.0), ("ag3", 0.3)):
        aflux, sflux, dd, du = photo.compute_flux_jax(g["tau"], g["ymix"], dev, g["dflux_u_prev"], ag0=ag0)
        assert rel(sflux.cpu().numpy(), g[f"{tag}_sflux"]) <= 1e-12
        assert rel_bin(dd.cpu().numpy(), g[f"{tag}_dflux_d"]) <= 1e-11
        assert rel_bin(du.cpu().numpy(), g[f"{tag}_dflux_u"]) <= 1e-11
        assert rel_bin(aflux.cpu().numpy(), g[f"{tag}_aflux"]) <= 1e-11
    J, JT = photo.compute_J_jax_flat(g["ag0_aflux"], dev)
    assert rel(J.cpu().numpy(), g["J_br"]) <= 1e-12
    assert rel(JT.cpu().numpy(), g["J_br_T"]) <= 1e-12


def test_update_k_with_J_active_branches():
    g = golden("photo.npz")
    ph = dict(_ph(g), branch_active=g["active"], branch_T_active=g["active_T"], f_diurnal=0.5)
    dev = photo.PhotoDevice(ph, g["y"].shape[0])
    k = torch.as_tensor(g["k"], device="cuda").clone()
    photo.update_k_with_J(k, g["ag0_aflux"], dev)
    assert rel(k.cpu().numpy(), g["k_new"]) <= 1e-12


def test_photo_update_config1_size():
    """nz=120, 2500 bins over 2-800 nm, 40 branches (the config-1 shapes)."""
    net = syn.make_network(0, 69, 700, n_photo=40)
    atm, extra = syn.make_atmosphere(0, net, nz=120)
    bins, din12 = syn.make_bins()
    ph = syn.make_photo(0, net, atm["Tco"], bins, din12)
    k = syn.make_rates(0, net, 120)
    prev = np.abs(np.random.default_rng(1).normal(0, 1, (121, bins.shape[0]))) * 1e3
    k_ref, aflux_ref, du_ref = op.photo_update(extra["y"], extra["ymix"], extra["dz"], k, ph, prev)
    dev = photo.PhotoDevice(ph, 120)
    kt = torch.as_tensor(k, device="cuda").clone()
    aflux, du = photo.photo_update(extra["y"], extra["ymix"], extra["dz"], kt, dev, prev)
    assert rel_bin(aflux.cpu().numpy(), aflux_ref) <= 1e-11
    assert rel_bin(du.cpu().numpy(), du_ref) <= 1e-11
    assert rel(kt.cpu().numpy(), k_ref) <= 1e-11
