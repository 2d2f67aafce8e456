"""Shared test setup.

``-m "not gpu"`` runs the oracle-vs-golden checks, the host-side logic and the
C-ABI export checks; ``-m gpu`` runs the CUDA parity tests through the C-ABI.
"""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_pkg(sub=None):
    """Import the package directory ``jax-vulcan_b200`` (or one of its modules)."""
    name = "jax-vulcan_b200" + ("." + sub if sub else "")
    return importlib.import_module(name)


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


STEP_CASES = ["plain", "moldiff", "full", "fixmask", "medium"]
ATM_KEYS = ["Kzz", "Dzz", "dzi", "vz", "Hpi", "Ti", "Tco", "g", "ms", "alpha", "M", "vm", "vs",
            "top_flux", "bot_flux", "bot_vdep", "gas_indx_mask"]
FLAG_KEYS = ["use_vm_mol", "use_settling", "use_topflux", "use_botflux"]


def golden_step(name):
    """Load a step fixture: (tables, atm dict, y, k, dt, fix_mask or None, fixture dict)."""
    g = golden(f"step_{name}.npz")
    net = load_pkg("network").parse_network_text(str(g["net_text"]))
    atm = {k: g["atm_" + k] for k in ATM_KEYS}
    atm.update({k: bool(g["atm_" + k]) for k in FLAG_KEYS})
    return net, atm, g["y"], g["k"], float(g["dt"]), g.get("fix_mask"), g


BODY_FIELDS = ["y", "y_prev", "ymix", "dt", "t", "delta", "accept_count", "retry_count", "atom_loss",
               "atom_loss_prev", "nega_count", "loss_count", "delta_count", "small_y", "nega_y", "rtol",
               "loss_criteria"]
BODY_OPT = ["use_fix_species", "non_gas", "hydro_partial", "zero_bot_row", "use_adapt_rtol", "loss_eps",
            "pos_cut"]


def golden_body():
    """Load the loop-body fixture: (tables, atm dict, compo, atom_ini, k,
    base params, {case: dict(inp, out, opt, gas, hist, fix_mask, fix_y)})."""
    g = golden("body.npz")
    net = load_pkg("network").parse_network_text(str(g["net_text"]))
    atm = {k: g["atm_" + k] for k in ATM_KEYS}
    atm.update({k: bool(g["atm_" + k]) for k in FLAG_KEYS})
    params = {k[6:]: g[k].item() for k in g if k.startswith("param_")}
    cases = {}
    for name in [str(n) for n in g["case_names"]]:
        inp = {f: (g[f"{name}_in_{f}"].item() if g[f"{name}_in_{f}"].ndim == 0 else g[f"{name}_in_{f}"])
               for f in BODY_FIELDS}
        out = {f: (g[f"{name}_out_{f}"].item() if g[f"{name}_out_{f}"].ndim == 0 else g[f"{name}_out_{f}"])
               for f in BODY_FIELDS}
        opt = dict(zip(BODY_OPT, g[f"{name}_opt"].tolist()))
        cases[name] = dict(inp=inp, out=out, opt=opt, gas=g[f"{name}_gas"], hist=g[f"{name}_hist"],
                           fix_mask=g[f"{name}_in_fix_mask"], fix_y=g[f"{name}_in_fix_y"])
    return net, atm, g["compo"], g["atom_ini"], g["k"], params, cases


def body_kwargs(case, params):
    """oracle.contract.attempt options and parameters of one body case."""
    o = case["opt"]
    p = dict(params, loss_eps=o["loss_eps"], pos_cut=o["pos_cut"], use_adapt_rtol=bool(o["use_adapt_rtol"]))
    kw = dict(gas=case["gas"] if o["non_gas"] else None, hydro_partial=bool(o["hydro_partial"]),
              zero_bot_row=bool(o["zero_bot_row"]))
    if o["use_fix_species"]:
        kw.update(fix_mask=case["fix_mask"], fix_y=case["fix_y"])
    return p, kw


@pytest.fixture
def pkg():
    return load_pkg()
