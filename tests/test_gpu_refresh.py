"""Atmosphere refresh and condensation on the GPU (``vb_atm_refresh``,
``vb_conden_rates``, ``vb_conden_relax``) against the reference's own
atm_refresh.py / conden.py output (``tests/golden/refresh.npz``) and the
oracle.

Tolerances: refresh 1e-14 relative (the per-layer mean molecular mass sums
species in order where NumPy's einsum may group them differently, and the
height integration carries that through ln and the running sum); escape
fluxes, condensation rows and the relaxation bit for bit (the same
element-wise expressions, NumPy's pairwise order for the gas sum).
"""
import numpy as np
import pytest
import torch

from conftest import golden, load_pkg
from oracle import refresh as orf

pytestmark = pytest.mark.gpu

jstep = load_pkg("jax_step")
ar = load_pkg("atm_refresh")
cd = load_pkg("conden")


def rel(a, b):
    a = np.asarray(a)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300), initial=0.0))


def blob_of(g, B=1, Tco=None, n_0=None):
    nz, ni = g["ymix"].shape
    Dzz = np.zeros((nz - 1, ni))
    Dzz[-1] = g["Dzz_top"]
    atm = dict(Kzz=np.ones(nz - 1), Dzz=Dzz, dzi=np.ones(nz - 1), vz=np.zeros(nz - 1), Hpi=np.ones(nz - 1),
               Ti=np.ones(nz - 1), Tco=g["Tco"], g=np.ones(nz), ms=g["ms"], alpha=np.zeros(ni), M=g["n_0"],
               vm=np.zeros((nz, ni)), vs=np.zeros((nz - 1, ni)), top_flux=g["top_flux"], bot_flux=np.zeros(ni),
               bot_vdep=np.zeros(ni), gas_indx_mask=g["gas"], use_vm_mol=False, use_settling=False,
               use_topflux=False, use_botflux=False)
    if B > 1:
        atm = {k: (np.stack([v] * B) if not isinstance(v, bool) else v) for k, v in atm.items()}
    if Tco is not None:
        atm["Tco"] = Tco
    if n_0 is not None:
        atm["M"] = n_0
    return jstep.pack_atm(jstep.atm_from_dict(atm)).contiguous()


def static_of(g):
    kb, Navo, gs, Rp, mf = g["consts"]
    return ar.AtmRefreshStatic(pico=g["pico"], mol_mass=g["mol_mass"], diff_esc_idx=g["esc"],
                               pref_indx=int(g["pref"]), zco_pref=0.0, gs=gs, Rp=Rp, kb=kb, Navo=Navo, max_flux=mf)


def test_refresh_matches_reference():
    g = golden("refresh.npz")
    nz, ni = g["ymix"].shape
    blob = blob_of(g)
    y = torch.as_tensor(g["y"][None], device="cuda")
    x = torch.as_tensor(g["ymix"][None], device="cuda")
    mu, Hp, dz, zco = ar.refresh(y, x, blob, static_of(g))
    f = ar.blob_fields(blob, nz, ni)
    for name, got in (("mu", mu[0]), ("Hp", Hp[0]), ("dz", dz[0]), ("zco", zco[0]), ("g", f["g"][0]),
                      ("dzi", f["dzi"][0]), ("Hpi", f["Hpi"][0])):
        e = rel(got.cpu().numpy(), g[name])
        assert e <= 1e-14, (name, e)
    tf = f["top_flux"][0].cpu().numpy()
    assert rel(tf, g["top_flux_new"]) <= 1e-14
    untouched = np.setdiff1d(np.arange(ni), g["esc"])
    assert np.array_equal(tf[untouched], g["top_flux"][untouched])
    mu1, g1, Hp1, dz1, zco1, dzi1, Hpi1 = ar.update_mu_dz_jax(g["ymix"], blob_of(g), static_of(g), y=g["y"])
    assert rel(zco1.cpu().numpy(), g["zco"]) <= 1e-14 and rel(Hpi1.cpu().numpy(), g["Hpi"]) <= 1e-14


def test_refresh_batch_against_oracle():
    """Three atmospheres with their own temperatures and mixing ratios in
    one launch, each against the oracle."""
    g = golden("refresh.npz")
    nz, ni = g["ymix"].shape
    rng = np.random.default_rng(5)
    T = np.stack([g["Tco"] * s for s in (1.0, 0.8, 1.3)])
    X = np.stack([g["ymix"] * rng.uniform(0.5, 1.5, g["ymix"].shape) for _ in range(3)])
    X /= X.sum(axis=2, keepdims=True)
    Y = X * g["n_0"][None, :, None]
    blob = blob_of(g, B=3, Tco=T)
    st = static_of(g)
    mu, Hp, dz, zco = ar.refresh(torch.as_tensor(Y, device="cuda"), torch.as_tensor(X, device="cuda"), blob, st)
    kb, Navo, gs, Rp, mf = g["consts"]
    f = ar.blob_fields(blob, nz, ni)
    for b in range(3):
        r = orf.update_mu_dz(X[b], T[b], g["pico"], g["mol_mass"], int(g["pref"]), 0.0, gs, Rp, kb, Navo)
        assert rel(zco[b].cpu().numpy(), r[4]) <= 1e-14 and rel(f["g"][b].cpu().numpy(), r[1]) <= 1e-14, b
        tf = orf.update_phi_esc(Y[b], r[1], r[2], g["top_flux"], T[b], g["Dzz_top"], g["ms"], g["esc"], kb, Navo, mf)
        assert rel(f["top_flux"][b].cpu().numpy(), tf) <= 1e-14, b


def test_conden_rates_and_relaxation_match_reference():
    g = golden("refresh.npz")
    nz, ni = g["ymix"].shape
    blob = blob_of(g)
    y = torch.as_tensor(g["y"][None], device="cuda").contiguous()
    x = torch.as_tensor(g["ymix"][None], device="cuda").contiguous()
    k = torch.as_tensor(g["k"][None], device="cuda").contiguous()
    st = cd.CondenStatic(conden_re_idx=g["re_idx"], conden_sp_idx=g["sp_idx"], Dg_per_re=g["Dg"][None],
                         sat_n_per_re=g["sat_n"][None], coeff_per_re=g["coeff"], atm_blob=blob, h2o_active=True,
                         h2o_idx=1, h2o_l_s_idx=2, h2o_Dg=g["Dg"][0], h2o_sat=g["sat_n"][0], h2o_m_over_rho_r2=0.7,
                         nh3_active=True, nh3_idx=4, nh3_l_s_idx=5, nh3_Dg=g["Dg"][1], nh3_sat=g["sat_n"][1],
                         nh3_m_over_rho_r2=0.3, nh3_conden_top=9)
    cd.update_conden_rates(k, y, st)
    assert np.array_equal(k[0].cpu().numpy(), g["k_new"])
    cd.apply_h2o_relax_jax(y, x, float(g["dt"]), st)
    assert np.array_equal(y[0].cpu().numpy(), g["y_h2o"]) and np.array_equal(x[0].cpu().numpy(), g["ymix_h2o"])
    cd.apply_nh3_relax_jax(y, x, float(g["dt"]), st)
    assert np.array_equal(y[0].cpu().numpy(), g["y_nh3"]) and np.array_equal(x[0].cpu().numpy(), g["ymix_nh3"])


def test_refresh_rejects_bad_arguments():
    import ctypes as C
    L = load_pkg("_lib").lib()
    g = golden("refresh.npz")
    p = static_of(g).params()
    p.pref_indx = 16
    dummy = C.c_void_p(16)  # never dereferenced: argument checks come first
    assert L.vb_atm_refresh(1, 16, 12, C.addressof(p), dummy, dummy, dummy, dummy, dummy, dummy, None, None, None,
                            None, None) == 1
    assert b"pref_indx" in L.vb_last_error()
    q = cd.VbRelaxParams()
    q.sp, q.sp_l_s = 3, 3
    assert L.vb_conden_relax(1, 16, 12, C.addressof(q), dummy, dummy, dummy, dummy, dummy, dummy, None) == 1
    torch.cuda.synchronize()
