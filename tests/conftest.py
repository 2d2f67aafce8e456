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


@pytest.fixture
def pkg():
    return load_pkg()
