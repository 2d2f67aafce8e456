"""CPU oracle for the photochemistry kernels (restatement of reference `photo.py`).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``smoke()`` and the CPU
baseline of ``bench.py``; never by the product path.

* ``compute_tau``    -> `photo.py:84-123`
* ``compute_flux``   -> `photo.py:126-245`
* ``compute_J``      -> `photo.py:309-351` (``_compute_J_inner``)
* ``update_k_with_J`` -> `photo.py:455-478`
* ``aflux_change``   -> `outer_loop.py:327-336`
"""
from __future__ import annotations

import numpy as np


def compute_tau(y, dz, ph):
    """Top-down optical depth tau[nz+1, nbin]; tau[nz] = 0. photo.py:84-123."""
    nz = y.shape[0]
    nbin = ph["absp_cross"].shape[1]
    if ph["absp_idx"].shape[0] > 0:
        a = np.einsum("js,sb->jb", y[:, ph["absp_idx"]], ph["absp_cross"]) * dz[:, None]
    else:
        a = np.zeros((nz, nbin))
    if ph["absp_T_idx"].shape[0] > 0:
        aT = np.sum(y[:, ph["absp_T_idx"]][:, :, None] * ph["absp_T_cross"].transpose(1, 0, 2),
                    axis=1) * dz[:, None]
        a = a + aT
    if ph["scat_idx"].shape[0] > 0:
        s = np.einsum("js,sb->jb", y[:, ph["scat_idx"]], ph["scat_cross"]) * dz[:, None]
        a = a + s
    tau_no_top = np.flip(np.cumsum(np.flip(a, axis=0), axis=0), axis=0)
    return np.concatenate([tau_no_top, np.zeros((1, nbin))], axis=0)


def compute_flux(tau, ymix, ph, dflux_u_prev):
    """Two-stream Eddington flux (ag0 = 0 and general branches). photo.py:126-245.

    Returns (aflux[nz,nbin], sflux[nz+1,nbin], dflux_d[nz+1,nbin], dflux_u[nz+1,nbin]).
    """
    sflux_top, bins = ph["sflux_top"], ph["bins"]
    mu_ang = -1.0 * ph["mu_zenith"]
    edd, ag0, hc = ph["edd"], ph["ag0"], ph["hc"]
    nz = tau.shape[0] - 1
    nbin = tau.shape[1]
    delta_tau = tau[:-1] - tau[1:]
    if ph["absp_idx"].shape[0] > 0:
        tot_abs = np.einsum("js,sb->jb", ymix[:, ph["absp_idx"]], ph["absp_cross"])
    else:
        tot_abs = np.zeros_like(delta_tau)
    if ph["absp_T_idx"].shape[0] > 0:
        tot_abs = tot_abs + np.sum(ymix[:, ph["absp_T_idx"]][:, :, None]
                                   * ph["absp_T_cross"].transpose(1, 0, 2), axis=1)
    if ph["scat_idx"].shape[0] > 0:
        tot_scat = np.einsum("js,sb->jb", ymix[:, ph["scat_idx"]], ph["scat_cross"])
    else:
        tot_scat = np.zeros_like(delta_tau)
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        w0 = tot_scat / np.maximum(tot_abs + tot_scat, 1e-300)
        w0 = np.where(np.isnan(w0), 0.0, w0)
        w0 = np.minimum(w0, 1.0 - 1e-8)
        sflux = sflux_top[None, :] * np.exp(tau / mu_ang)
        dir_flux = sflux * (-mu_ang)
        if ag0 == 0:
            tran = np.exp(-1.0 / edd * (1.0 - w0) ** 0.5 * delta_tau)
            zeta_p = 0.5 * (1.0 + (1.0 - w0) ** 0.5)
            zeta_m = 0.5 * (1.0 - (1.0 - w0) ** 0.5)
            ll = -1.0 * w0 / (1.0 / mu_ang ** 2 - 1.0 / edd ** 2 * (1.0 - w0))
            g_p = 0.5 * (ll * (1.0 / edd + 1.0 / mu_ang))
            g_m = 0.5 * (ll * (1.0 / edd - 1.0 / mu_ang))
        else:
            tran = np.exp(-1.0 / edd * ((1.0 - w0 * ag0) * (1.0 - w0)) ** 0.5 * delta_tau)
            zeta_p = 0.5 * (1.0 + ((1.0 - w0) / (1.0 - w0 * ag0)) ** 0.5)
            zeta_m = 0.5 * (1.0 - ((1.0 - w0) / (1.0 - w0 * ag0)) ** 0.5)
            ll = ((1.0 - w0) * (1.0 - w0 * ag0) - 1.0) / (
                1.0 / mu_ang ** 2 - 1.0 / edd ** 2 * (1.0 - w0) * (1.0 - w0 * ag0))
            g_p = 0.5 * (ll * (1.0 / edd + 1.0 / (mu_ang * (1.0 - w0 * ag0)))
                         + w0 * ag0 * mu_ang / (1.0 - w0 * ag0))
            g_m = 0.5 * (ll * (1.0 / edd - 1.0 / (mu_ang * (1.0 - w0 * ag0)))
                         - w0 * ag0 * mu_ang / (1.0 - w0 * ag0))
        ll = np.clip(ll, -1e10, 1e10)
        chi = zeta_m ** 2 * tran ** 2 - zeta_p ** 2
        xi = zeta_p * zeta_m * (1.0 - tran ** 2)
        phi = (zeta_m ** 2 - zeta_p ** 2) * tran
        i_u = phi * g_p * dir_flux[:-1] - (xi * g_m + chi * g_p) * dir_flux[1:]
        i_d = phi * g_m * dir_flux[1:] - (chi * g_m + xi * g_p) * dir_flux[:-1]
        dflux_d = np.zeros((nz + 1, nbin))
        for j in range(nz - 1, -1, -1):                                    # photo.py:210-223
            dflux_d[j] = (1.0 / chi[j]) * (phi[j] * dflux_d[j + 1] - xi[j] * dflux_u_prev[j]
                                           + i_d[j] / mu_ang)
        dflux_u = np.zeros((nz + 1, nbin))
        for j in range(1, nz + 1):                                         # photo.py:227-236
            dflux_u[j] = (1.0 / chi[j - 1]) * (phi[j - 1] * dflux_u[j - 1] - xi[j - 1] * dflux_d[j]
                                               + i_u[j - 1] / mu_ang)
        ave_dir = 0.5 * (sflux[:-1] + sflux[1:])
        tot_flux = ave_dir + 0.5 * (dflux_u[:-1] + dflux_u[1:] + dflux_d[1:] + dflux_d[:-1]) / edd
        aflux = tot_flux / (hc / bins[None, :])
    return aflux, sflux, dflux_d, dflux_u


def compute_J(aflux, ph):
    """Two-resolution trapezoid J-rates -> (J_br[n_br,nz], J_br_T[n_br_T,nz]). photo.py:309-351."""
    d = ph["din12_indx"]
    dbin1, dbin2 = ph["dbin1"], ph["dbin2"]
    cross_J, cross_J_T = ph["cross_J"], ph["cross_J_T"]
    nz = aflux.shape[0]
    f1, f2 = aflux[:, :d], aflux[:, d:]
    if cross_J.shape[0] > 0:
        c1, c2 = cross_J[:, :d], cross_J[:, d:]
        J1 = np.einsum("jb,nb->nj", f1, c1) * dbin1
        J1 = J1 - 0.5 * (f1[:, 0][None] * c1[:, 0][:, None] + f1[:, -1][None] * c1[:, -1][:, None]) * dbin1
        J2 = np.einsum("jb,nb->nj", f2, c2) * dbin2
        J2 = J2 - 0.5 * (f2[:, 0][None] * c2[:, 0][:, None] + f2[:, -1][None] * c2[:, -1][:, None]) * dbin2
        J_br = J1 + J2
    else:
        J_br = np.zeros((0, nz))
    if cross_J_T.shape[0] > 0:
        t1, t2 = cross_J_T[:, :, :d], cross_J_T[:, :, d:]
        JT1 = np.sum(f1[None] * t1, axis=2) * dbin1
        JT1 = JT1 - 0.5 * (f1[:, 0][None] * t1[:, :, 0] + f1[:, -1][None] * t1[:, :, -1]) * dbin1
        JT2 = np.sum(f2[None] * t2, axis=2) * dbin2
        JT2 = JT2 - 0.5 * (f2[:, 0][None] * t2[:, :, 0] + f2[:, -1][None] * t2[:, :, -1]) * dbin2
        J_br_T = JT1 + JT2
    else:
        J_br_T = np.zeros((0, nz))
    return J_br, J_br_T


def update_k_with_J(k_arr, J_br, J_br_T, re_idx, active, re_T_idx, active_T, f_diurnal):
    """k_arr[re_idx] = J * f_diurnal for active branches. photo.py:455-478."""
    Js = J_br * f_diurnal
    JTs = J_br_T * f_diurnal
    safe = np.where(np.asarray(active, bool)[:, None], Js, k_arr[0][None, :])
    safe_T = np.where(np.asarray(active_T, bool)[:, None], JTs, k_arr[0][None, :])
    idx = np.concatenate([re_idx, re_T_idx])
    vals = np.concatenate([safe, safe_T], axis=0)
    out = k_arr.copy()
    out[idx] = vals
    return out


def photo_update(y, ymix, dz, k_arr, ph, dflux_u_prev):
    """tau -> flux -> J -> k rows, the in-loop photo branch (reference
    `outer_loop.py:283-350`). Returns (k_new, aflux, dflux_u)."""
    tau = compute_tau(y, dz, ph)
    aflux, sflux, dflux_d, dflux_u = compute_flux(tau, ymix, ph, dflux_u_prev)
    J_br, J_br_T = compute_J(aflux, ph)
    nb, nbT = J_br.shape[0], J_br_T.shape[0]
    k_new = update_k_with_J(k_arr, J_br, J_br_T, ph["branch_re_idx"], np.ones(nb, bool),
                            ph["branch_T_re_idx"], np.ones(nbT, bool), ph["f_diurnal"])
    return k_new, aflux, dflux_u


def aflux_change(aflux_new, aflux_old, flux_atol):
    """Largest relative change of the actinic flux over the entries above
    ``flux_atol``; 0 when none is (reference `outer_loop.py:327-336`)."""
    mask = aflux_new > flux_atol
    if not mask.any():
        return 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.where(mask, np.abs(aflux_new - aflux_old) / np.maximum(np.abs(aflux_new), 1e-300), 0.0)
    return float(np.max(ratio))
