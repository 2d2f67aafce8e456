"""Build ``libvulcan_b200.so`` in-tree with nvcc for sm_100a.

The chemistry/diffusion unit is compiled with ``--fmad=false`` so its sums
and products round exactly like the reference's element-wise expressions; the
solver units keep fused multiply-add.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvulcan_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
          "--expt-relaxed-constexpr"]
UNITS = {
    "vb_api.cu": [],
    "vb_thomas.cu": [],
    "vb_chem.cu": ["--fmad=false"],
    "vb_photo.cu": ["--fmad=false"],
    "vb_adjoint.cu": [],
    "vb_control.cu": ["--fmad=false"],
    "vb_mixed.cu": [],
    "vb_rates.cu": ["--fmad=false"],
    "vb_refresh.cu": ["--fmad=false"],
}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False, ptxas_v=False):
    """Compile every unit and link the shared library. Returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(INCLUDE, "vulcan_b200.h"))
    objs, cmds = [], []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + headers + [__file__]):
            cmds.append([nvcc()] + ARCH + COMMON + extra + (["-Xptxas", "-v"] if ptxas_v else []) +
                        ["-c", src, "-o", obj])
    # the units compile independently: one nvcc process per unit, in parallel
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd))
        for f in [pool.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            f.result()
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_v="-v" in sys.argv)
