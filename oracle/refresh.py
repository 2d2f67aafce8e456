"""CPU oracle for the atmosphere refresh and the condensation kernels
(restatement of reference `atm_refresh.py` and `conden.py`).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``; never by the product path.

* ``update_mu_dz``        -> `atm_refresh.py:36-100`: mean molecular mass,
  then the hydrostatic integration upward from the reference layer and
  downward below it (g, Hp, dz, zco), and the interface means dzi, Hpi
* ``update_phi_esc``      -> `atm_refresh.py:103-122`: diffusion-limited
  escape flux at the top, floored at -max_flux
* ``update_conden_rates`` -> `conden.py:55-71`
* ``apply_relax``         -> `conden.py:74-160` (H2O without, NH3 with the
  condensation clamp to layers <= conden_top and the clip of the condensate)
"""
from __future__ import annotations

import numpy as np


def update_mu_dz(ymix, Tco, pico, mol_mass, pref_indx, zco_pref, gs, Rp, kb, Navo):
    nz = Tco.shape[0]
    mu = np.einsum("zi,i->z", ymix, mol_mass)
    g, Hp, dz = np.zeros(nz), np.zeros(nz), np.zeros(nz)
    zco = np.zeros(nz + 1)
    zco[pref_indx] = zco_pref
    z = np.float64(zco_pref)
    for i in range(pref_indx, nz):
        gi = gs if i == pref_indx else gs * (Rp / (Rp + z)) ** 2
        Hpi = kb * Tco[i] / (mu[i] / Navo * gi)
        dzi = Hpi * np.log(pico[i] / pico[i + 1])
        z = z + dzi
        g[i], Hp[i], dz[i], zco[i + 1] = gi, Hpi, dzi, z
    z = np.float64(zco_pref)
    for i in range(pref_indx - 1, -1, -1):
        gi = gs * (Rp / (Rp + z)) ** 2
        Hpi = kb * Tco[i] / (mu[i] / Navo * gi)
        dzi = Hpi * np.log(pico[i] / pico[i + 1])
        z = z - dzi
        g[i], Hp[i], dz[i], zco[i] = gi, Hpi, dzi, z
    return mu, g, Hp, dz, zco, 0.5 * (dz[:-1] + dz[1:]), 0.5 * (Hp[:-1] + Hp[1:])


def update_phi_esc(y, g, Hp, top_flux, Tco, Dzz_top, ms, esc_idx, kb, Navo, max_flux):
    out = np.array(top_flux, dtype=np.float64, copy=True)
    e = np.asarray(esc_idx)
    flux = -Dzz_top[e] * y[-1, e] * (1.0 / Hp[-1] - ms[e] * g[-1] / (Navo * kb * Tco[-1]))
    out[e] = np.maximum(flux, -max_flux)
    return out


def update_conden_rates(k, y, re_idx, sp_idx, Dg, sat_n, coeff):
    rate = Dg * coeff[:, None] * (y[:, sp_idx].T - sat_n)
    k = k.copy()
    k[re_idx] = np.maximum(rate, 0.0)
    k[np.asarray(re_idx) + 1] = np.maximum(-rate, 0.0)
    return k


def apply_relax(y, ymix, dt, sp, sp_l_s, Dg, sat, m_over_rho_r2, n_0, gas_mask, conden_top=None):
    """One species' implicit-Euler cold-trap relaxation; ``conden_top`` given
    (NH3) clamps condensation to layers <= conden_top and clips the
    condensate at zero."""
    denom = Dg * m_over_rho_r2 * (y[:, sp] - sat)
    denom = np.where(np.abs(denom) < 1e-300, 1e-300, denom)
    tau = 1.0 / denom
    sat_mix = sat / n_0
    y_conden = (ymix[:, sp] + dt / tau * sat_mix) / (1.0 + dt / tau)
    ice_loss = np.minimum(y[:, sp_l_s], (y[:, sp] - sat) * dt / tau)
    conden = tau > 0
    if conden_top is not None:
        conden = conden & (np.arange(y.shape[0]) <= conden_top)
    d_c = np.where(conden, ymix[:, sp] - y_conden, 0.0)
    d_e = np.where(tau < 0, ice_loss / n_0, 0.0)
    x = ymix.copy()
    x[:, sp_l_s] = x[:, sp_l_s] + d_c
    x[:, sp] = x[:, sp] + (-d_c)
    x[:, sp] = x[:, sp] + d_e
    x[:, sp_l_s] = x[:, sp_l_s] + (-d_e)
    if conden_top is not None:
        x[:, sp_l_s] = np.maximum(x[:, sp_l_s], 0.0)
    ysum = np.sum(np.where(np.asarray(gas_mask, bool)[None, :], y, 0.0), axis=1, keepdims=True)
    return x * ysum, x
