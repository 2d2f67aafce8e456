"""The C-ABI library loads and exports every symbol the header declares (CPU only:
no compute call is made without a GPU)."""
import os
import re
import subprocess

from conftest import ROOT, load_pkg

HEADER = os.path.join(ROOT, "include", "vulcan_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vb_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    lib = load_pkg("_lib")
    path = lib.LIB_PATH
    assert os.path.exists(path), "build() has not produced the library"
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\s[TW]\s+(vb_[A-Za-z0-9_]+)$", out, flags=re.M))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_ctypes_binding_covers_header():
    lib = load_pkg("_lib")
    assert sorted(lib.SIGNATURES) == declared_symbols()
    h = lib.lib()
    assert h.vb_version() >= 1
    # size queries are host-only
    assert h.vb_bt_factor_bytes(2, 10, 69) > 0
    assert h.vb_ros2_workspace_bytes(2, 10, 69, None) > 0
