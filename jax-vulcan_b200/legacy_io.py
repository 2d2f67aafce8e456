"""``.vul`` output of one atmosphere of the device loop (reference
`legacy_io.py:429-790`).

``vul_dicts`` builds the three top-level dicts of the reference's pickle
(`variable`, `atm`, `parameter`) from host copies of the loop carry, with the
keys, shapes and types the reference writer publishes
(`_synthesize_save_dicts`) and its comparison tool reads (`tests/compare_vul.py`:
species, nr, y_ini, y, ymix, t, dt, longdy, atom_loss). ``write_vul`` pickles
them (protocol 4, as the reference). Keys of features this package does not
run (ions, the saved evolution, condensation bookkeeping, plotting colours)
are left out; ``atom_conden`` is published as zeros, as the reference does.
"""
from __future__ import annotations

import pickle

import numpy as np


def _host(x):
    if x is None:
        return None
    if hasattr(x, "detach"):
        x = x.detach().cpu().numpy()
    return np.asarray(x)


def vul_dicts(species, k, snap, b=0, y_ini=None, compo=None, atom_order=None, atom_ini=None, conv=None, atm=None,
              Rf=None, photo=None, photo_carry=None):
    """The (variable, atm, parameter) dicts of atmosphere ``b``.

    ``species``: species names; ``k`` [nr+1, nz] or [B, nr+1, nz]; ``snap``:
    ``LoopState.snapshot()`` (or a dict with the same fields); ``conv``:
    ``LoopState.conv_host()`` records; ``compo`` [ni, n_atoms] with
    ``atom_order`` names and ``atom_ini`` [n_atoms] (or [B, n_atoms]) for the
    atom dicts; ``atm``: dict of the atmosphere arrays, batched ([B, ...])
    when the carry is; ``Rf``: forward row -> reaction text; ``photo``: the photo table
    dict (bins, dbin1, dbin2); ``photo_carry``: ``photo.PhotoCarry``."""
    y_all = _host(snap["y"])
    y = y_all[b] if y_all.ndim == 3 else y_all
    ymix_all = _host(snap["ymix"])
    ymix = ymix_all[b] if ymix_all.ndim == 3 else ymix_all
    ka = _host(k)
    ka = ka[b] if ka.ndim == 3 else ka

    def scal(name):
        v = np.asarray(snap[name])
        return v.reshape(-1)[b] if v.ndim else v

    var = {"species": list(species), "nr": int(ka.shape[0] - 1),
           "k": {i: ka[i].copy() for i in range(1, ka.shape[0])},
           "y": np.asarray(y, np.float64), "ymix": np.asarray(ymix, np.float64),
           "t": float(scal("t")), "dt": float(np.asarray(snap["dt"]).reshape(-1)[b])}
    if conv is not None:
        c = conv[b] if np.ndim(conv) else conv
        var["longdy"] = float(c["longdy"])
        var["longdydt"] = float(c["longdydt"])
    if y_ini is not None:
        yi = _host(y_ini)
        var["y_ini"] = np.asarray(yi[b] if yi.ndim == 3 else yi, np.float64)
    if compo is not None and atom_order is not None:
        cm = _host(compo)
        asum = np.einsum("zi,ia->a", y, cm)
        ai = _host(atom_ini) if atom_ini is not None else asum
        ai = ai[b] if np.ndim(ai) == 2 else ai
        al = np.asarray(snap["atom_loss"])
        al = al[b] if al.ndim == 2 else al
        var["atom_ini"] = {sp: float(ai[i]) for i, sp in enumerate(atom_order)}
        var["atom_sum"] = {sp: float(asum[i]) for i, sp in enumerate(atom_order)}
        var["atom_loss"] = {sp: float(al[i]) for i, sp in enumerate(atom_order)}
        var["atom_conden"] = {sp: 0.0 for sp in atom_order}
    if photo_carry is not None:
        var["tau"] = _host(photo_carry.tau)[b].astype(np.float64)
        var["sflux"] = _host(photo_carry.sflux)[b].astype(np.float64)
        var["aflux"] = _host(photo_carry.aflux)[b].astype(np.float64)
        if conv is not None:
            var["aflux_change"] = float((conv[b] if np.ndim(conv) else conv)["aflux_change"])
    if photo is not None:
        bins = np.asarray(photo["bins"], np.float64)
        var.update(nbin=int(bins.shape[0]), bins=bins, dbin1=float(photo["dbin1"]), dbin2=float(photo["dbin2"]))
    if Rf is not None:
        var["Rf"] = dict(Rf)

    atm_save = {}
    for name, v in (atm or {}).items():
        if isinstance(v, (bool, np.bool_)):
            atm_save[name] = bool(v)
            continue
        a = _host(v)
        atm_save[name] = a[b] if (y_all.ndim == 3 and a.ndim >= 1) else a
    atm_save["conden_min_lev"] = {}

    para = {"count": int(scal("accept_count")), "nega_count": int(scal("nega_count")),
            "loss_count": int(scal("loss_count")), "delta_count": int(scal("delta_count")),
            "delta": float(scal("delta")), "small_y": float(scal("small_y")), "nega_y": float(scal("nega_y")),
            "end_case": 0, "solver_str": "solver", "switch_final_photo_frq": False,
            "where_varies_most": np.zeros_like(var["y"]), "pic_count": 0, "fix_species_start": False}
    if conv is not None:
        c = conv[b] if np.ndim(conv) else conv
        para["switch_final_photo_frq"] = bool(c["is_final_photo_frq"])
        para["end_case"] = 1 if int(c["done"]) else 0
    return var, atm_save, para


def write_vul(path, *args, **kw):
    """Write the ``.vul`` pickle of one atmosphere (arguments as ``vul_dicts``)."""
    var, atm_save, para = vul_dicts(*args, **kw)
    with open(path, "wb") as f:
        pickle.dump({"variable": var, "atm": atm_save, "parameter": para}, f, protocol=4)
    return path
