"""CPU oracle for the rate-constant build (restatement of reference `rates.py`
and `gibbs.py`).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``; never by the product path.

* ``compute_forward_k`` -> `rates.py:61-125` (modified Arrhenius, Lindemann
  falloff, the hardcoded Troe of `OH + CH3 + M -> CH3OH + M` `:36-58`; photo,
  ion, condensation and radiative slots stay zero)
* ``apply_lowT_caps``   -> `rates.py:141-166`
* ``apply_remove_list`` -> `rates.py:169-181`
* ``gibbs_sp_vector``   -> `gibbs.py:41-73` (NASA-9 g/RT, low branch below 1000 K)
* ``K_eq_array``        -> `gibbs.py:76-125`
* ``fill_reverse_k``    -> `gibbs.py:128-150`
* ``build_rate_array``  -> `rates.py:184-208`

Every function also accepts a complex temperature ``T + i h`` (branch tests
use the real part), so ``dk_dT`` gets the temperature derivative of the
whole build by complex-step differentiation, exact to rounding.
``net`` is this package's ``NetworkTables`` (rate columns and section flags).
"""
from __future__ import annotations

import numpy as np

KB = 1.38064852e-16          # erg/K (reference phy_const.kb)
CORR = KB / 1.0e6            # gibbs.py:11-12

SPECIAL_OH_CH3 = "OH + CH3 + M -> CH3OH + M"
CAP_CH3 = "H + CH3 + M -> CH4 + M"
CAP_C2H4 = "H + C2H4 + M -> C2H5 + M"
CAP_C2H5 = "H + C2H5 + M -> C2H6 + M"


def _re(x):
    return np.real(x)


def arrhenius(a, n, E, T):
    """a T^n exp(-E/T) (rates.py:36-38)."""
    return a * T ** n * np.exp(-E / T)


def troe_oh_ch3(T, M):
    """Hardcoded Troe falloff of OH + CH3 + M -> CH3OH + M (rates.py:41-58)."""
    k0 = 1.932e3 * T ** -9.88 * np.exp(-7544.0 / T) + 5.109e-11 * T ** -6.25 * np.exp(-1433.0 / T)
    kinf = 1.031e-10 * T ** -0.018 * np.exp(16.74 / T)
    Fc = 0.1855 * np.exp(-T / 155.8) + 0.8145 * np.exp(-T / 1675.0) + np.exp(-4531.0 / T)
    nn = 0.75 - 1.27 * np.log(Fc)
    ff = np.exp(np.log(Fc) / (1.0 + (np.log(k0 * M / kinf) / nn) ** 2))
    return k0 / (1.0 + k0 * M / kinf) * ff


def compute_forward_k(net, T, M):
    """Forward rate constants k[nr+1, nz]; reverse and runtime-filled slots 0."""
    T = np.asarray(T)
    k = np.zeros((net.nr + 1, T.shape[0]), dtype=T.dtype if np.iscomplexobj(T) else np.float64)
    for i in range(1, net.nr + 1, 2):
        if not net.is_forward[i] or net.is_photo[i] or net.is_ion[i] or net.is_conden[i] or net.is_radiative[i]:
            continue
        if net.is_special[i]:
            if net.Rf.get(i, "").strip() == SPECIAL_OH_CH3:
                k[i] = troe_oh_ch3(T, M)
            elif net.a[i] != 0.0:
                k[i] = arrhenius(net.a[i], net.n[i], net.E[i], T)
            continue
        if net.has_kinf[i]:
            k0 = arrhenius(net.a[i], net.n[i], net.E[i], T)
            kinf = arrhenius(net.a_inf[i], net.n_inf[i], net.E_inf[i], T)
            k[i] = k0 / (1.0 + k0 * M / kinf)
        else:
            k[i] = arrhenius(net.a[i], net.n[i], net.E[i], T)
    return k


def apply_lowT_caps(net, k, T, M):
    """The three low-temperature caps on the forward rows (rates.py:141-166)."""
    k = k.copy()
    Tr = _re(T)
    for i in range(1, net.nr + 1, 2):
        if not net.is_forward[i]:
            continue
        rf = net.Rf.get(i, "")
        if rf == CAP_CH3:
            k0 = 6.0e-29
            kinf = 2.06e-10 * T ** -0.4
            k[i] = np.where(Tr <= 277.5, k0 / (1.0 + k0 * M / kinf), k[i])
        elif rf == CAP_C2H4:
            k[i] = np.where(Tr <= 300.0, 3.7e-30, k[i])
        elif rf == CAP_C2H5:
            k[i] = np.where(Tr <= 200.0, 2.49e-27, k[i])
    return k


def apply_remove_list(net, k, remove_list):
    """Zero the listed rows, no forward/reverse pairing (rates.py:169-181)."""
    k = k.copy()
    for i in remove_list or ():
        if 0 <= int(i) <= net.nr:
            k[int(i)] = 0.0
    return k


def gibbs_sp_vector(coeffs, T):
    """g/(RT) per species and layer [ni, nz] from NASA-9 coefficients
    [ni, 2, 10] (gibbs.py:41-73): H/RT - S/R of the low branch below 1000 K,
    else of the high branch."""
    T = np.asarray(T)[None, :]

    def branch(a):
        h = (-a[:, 0:1] / T ** 2 + a[:, 1:2] * np.log(T) / T + a[:, 2:3] + a[:, 3:4] * T / 2.0
             + a[:, 4:5] * T ** 2 / 3.0 + a[:, 5:6] * T ** 3 / 4.0 + a[:, 6:7] * T ** 4 / 5.0 + a[:, 8:9] / T)
        s = (-a[:, 0:1] / T ** 2 / 2.0 - a[:, 1:2] / T + a[:, 2:3] * np.log(T) + a[:, 3:4] * T
             + a[:, 4:5] * T ** 2 / 2.0 + a[:, 5:6] * T ** 3 / 3.0 + a[:, 6:7] * T ** 4 / 4.0 + a[:, 9:10])
        return h - s

    return np.where(_re(T) < 1000.0, branch(coeffs[:, 0, :]), branch(coeffs[:, 1, :]))


def K_eq_array(net, g, T):
    """Equilibrium constants of the forward rows [nr+1, nz] (gibbs.py:76-125):
    exp(sum st g(reactants) - sum st g(products)) (CORR T)^(dn); 1 where the
    row has no thermal reverse."""
    T = np.asarray(T)
    K = np.ones((net.nr + 1, T.shape[0]), dtype=g.dtype)
    gp = np.concatenate([g, np.zeros((1, T.shape[0]), dtype=g.dtype)], axis=0)
    for i in range(1, net.nr + 1, 2):
        if not net.is_forward[i] or i + 1 >= net.stop_rev_indx:
            continue
        if net.is_photo[i] or net.is_ion[i] or net.is_conden[i] or net.is_radiative[i]:
            continue
        rs = np.zeros(T.shape[0], dtype=g.dtype)
        for sp, st in zip(net.reactant_idx[i], net.reactant_stoich[i]):
            if st != 0.0:
                rs = rs + st * gp[sp]
        ps = np.zeros(T.shape[0], dtype=g.dtype)
        for sp, st in zip(net.product_idx[i], net.product_stoich[i]):
            if st != 0.0:
                ps = ps + st * gp[sp]
        dn = float(net.reactant_stoich[i].sum()) - float(net.product_stoich[i].sum())
        K[i] = np.exp(rs - ps)
        if dn != 0.0:
            K[i] = K[i] * (CORR * T) ** dn
    return K


def fill_reverse_k(net, k, K):
    """Reverse rows k[i] = k[i-1] / K[i-1] for even i < stop_rev_indx (0 where
    K <= 0); even rows past stop_rev_indx zero (gibbs.py:128-150)."""
    k = k.copy()
    for i in range(2, net.stop_rev_indx, 2):
        Ki = K[i - 1]
        with np.errstate(divide="ignore", invalid="ignore"):
            k[i] = np.where(_re(Ki) > 0, k[i - 1] / Ki, 0.0)
    for i in range(net.stop_rev_indx + 1, net.nr + 1, 2):
        k[i] = 0.0
    return k


def build_rate_array(net, coeffs, T, M, lowT_caps=False, remove_list=None):
    """Forward -> (low-T caps) -> reverse from NASA-9 Gibbs -> removal
    (rates.py:184-208)."""
    k = compute_forward_k(net, T, M)
    if lowT_caps:
        k = apply_lowT_caps(net, k, T, M)
    k = fill_reverse_k(net, k, K_eq_array(net, gibbs_sp_vector(coeffs, T), T))
    return apply_remove_list(net, k, remove_list)


def dk_dT(net, coeffs, T, M, lowT_caps=False, remove_list=None, h=1e-30):
    """Temperature derivative of ``build_rate_array`` at fixed M, by complex
    step: Im k(T + i h) / h (no subtractive cancellation)."""
    kc = build_rate_array(net, coeffs, np.asarray(T, np.float64) + 1j * h, M, lowT_caps, remove_list)
    return np.imag(kc) / h
