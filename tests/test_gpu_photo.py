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


def photo_batch_case(nbin_max=402.0, nz=12):
    net = syn.make_network(7, 30, 185, n_photo=10)
    atm, extra = syn.make_atmosphere(7, net, nz=nz)
    bins, din12 = syn.make_bins(bin_max=nbin_max)
    ph = syn.make_photo(7, net, atm["Tco"], bins, din12)
    return net, atm, extra, ph


def test_photo_branch_masked_with_aflux_change():
    """vb_photo_update on three atmospheres with due = [1, 0, 1]: the due
    ones bit for bit equal to the separate tau / flux / J calls (which read
    the previous upward flux from another buffer: the in-place update of
    dflux_u must not change a bit) and against the oracle (tau -> flux -> J ->
    k rows, aflux change against the aflux held on entry); the other bit for
    bit untouched. Tolerances as above, except the upward flux: on this grid
    (12 optically thick layers) a relative change of 4e-16 in y moves dflux_u
    by 1e-11 of its bin maximum (measured with the oracle), so the 1e-12 of
    tau allows ~1e-8 there. The aflux change (a ratio of differences of order
    1e-2 .. 1) within 1e-9 relative."""
    net, atm, extra, ph = photo_batch_case()
    nz, nbin = extra["y"].shape[0], ph["bins"].shape[0]
    rng = np.random.default_rng(3)
    ys = [extra["y"] * s for s in (1.0, 0.5, 2.0)]
    ymix = extra["ymix"]
    k0 = syn.make_rates(7, net, nz)
    prev = np.abs(rng.normal(0, 1, (3, nz + 1, nbin))) * 1e3
    dev = photo.PhotoDevice(ph, nz)
    carry = photo.PhotoCarry(dev, 3, nz, dflux_u=prev)
    refs = [op.photo_update(ys[b], ymix, extra["dz"], k0, ph, prev[b]) for b in range(3)]
    old = np.stack([refs[0][1] * (1.0 + 0.05 * rng.standard_normal((nz, nbin))),
                    np.full((nz, nbin), 7.0), np.zeros((nz, nbin))])
    carry.aflux.copy_(torch.as_tensor(old))
    loop = load_pkg("outer_loop")
    rec = np.zeros(3, loop.CONV_DTYPE)
    rec["aflux_change"] = [-1.0, 0.25, -1.0]
    conv = torch.from_numpy(rec.view(np.uint8).copy()).cuda()
    k = torch.as_tensor(np.stack([k0] * 3), device="cuda").contiguous()
    due = torch.tensor([1, 0, 1], dtype=torch.int32, device="cuda")
    y = torch.as_tensor(np.stack(ys), device="cuda")
    x = torch.as_tensor(np.stack([ymix] * 3), device="cuda")
    photo.photo_branch(carry, y, x, extra["dz"], k, dev, due=due, flux_atol=1.0, conv=conv)
    got = conv.cpu().numpy().view(loop.CONV_DTYPE)
    for b in (0, 2):
        k1 = torch.as_tensor(k0, device="cuda").clone()
        a1, du1 = photo.photo_update(ys[b], ymix, extra["dz"], k1, dev, prev[b])
        assert torch.equal(carry.aflux[b], a1) and torch.equal(carry.dflux_u[b], du1) and torch.equal(k[b], k1)
        k_ref, a_ref, du_ref = refs[b]
        assert rel_bin(carry.aflux[b].cpu().numpy(), a_ref) <= 1e-11
        assert rel_bin(carry.dflux_u[b].cpu().numpy(), du_ref) <= 1e-8
        assert rel(k[b].cpu().numpy(), k_ref) <= 1e-11
        want = op.aflux_change(a_ref, old[b], 1.0)
        assert abs(got["aflux_change"][b] - want) <= 1e-9 * abs(want), (b, got["aflux_change"][b], want)
    assert got["aflux_change"][2] == 1.0          # from zeros: every entry above flux_atol changed fully
    assert got["aflux_change"][1] == 0.25
    assert np.array_equal(carry.aflux[1].cpu().numpy(), old[1])
    assert np.array_equal(carry.dflux_u[1].cpu().numpy(), prev[1])
    assert np.array_equal(k[1].cpu().numpy(), k0)
