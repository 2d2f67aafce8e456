"""Autotuner of the step's launch shapes.

The reference batches atmospheres with ``jax.vmap`` and leaves kernel shapes
to XLA (reference `examples/batched_run.py:60-63`). Here the shapes are
chosen by timing: for every network group of a batch (its species count,
reaction count, atmosphere count and layer total), each candidate
``VbTuning`` (factor kernel, factor CTAs per SM where both variants exist,
depth of the sweeps' bulk-copy ring) is applied to the network and the
group's Ros2 step is timed with CUDA events on the device; the fastest is
kept. Choices are cached in a JSON file keyed by the group's shape and the
GPU name, and ``MultiNetworkBatch(tuning=...)`` applies a cache before it
captures its graph.
"""
from __future__ import annotations

import ctypes as C
import itertools
import json
import os

import torch

from . import _lib


class VbTuning(C.Structure):
    _fields_ = [("factor_kernel", C.c_int32), ("factor_ctas", C.c_int32), ("sweep_stages", C.c_int32),
                ("streams", C.c_int32), ("stage1_layers", C.c_int32), ("reserved", C.c_int32)]


FIELDS = ("factor_kernel", "factor_ctas", "sweep_stages", "streams", "stage1_layers")


def set_tuning(net, tuning: dict) -> None:
    """Apply a tuning (dict with the FIELDS; missing fields automatic) to a network."""
    t = VbTuning(*(int(tuning.get(f, 0)) for f in FIELDS), 0)
    _lib.check(_lib.lib().vb_net_set_tuning(net.handle, C.addressof(t)), "vb_net_set_tuning")


def get_tuning(net) -> dict:
    t = VbTuning()
    _lib.check(_lib.lib().vb_net_get_tuning(net.handle, C.addressof(t)), "vb_net_get_tuning")
    return {f: int(getattr(t, f)) for f in FIELDS}


def candidates(ni: int, split: bool = False):
    """Candidate tunings of a network with ni species; ``split``: also the
    two-stream step (uniform batches only)."""
    ctas = (1, 2) if 64 < ni <= 72 else (0,)
    kernels = (1, 2, 3, 4) if 64 < ni <= 72 else (1, 2, 3)   # 4: the paired kernel (65-72 species)
    streams = (1, 2) if split else (1,)
    for fk, fc, ss, sn, s1 in itertools.product(kernels, ctas, (2, 3), streams, (1, 2)):
        if fk == 4 and fc == 2:
            continue   # one paired CTA per SM holds two atmospheres: no CTA-count choice
        yield {"factor_kernel": fk, "factor_ctas": fc, "sweep_stages": ss, "streams": sn, "stage1_layers": s1}


def group_key(net, batch: int, layers: int) -> str:
    gpu = torch.cuda.get_device_name() if torch.cuda.is_available() else "none"
    return f"{gpu}|ni={net.ni}|nr={net.nr}|batch={batch}|layers={layers}"


def time_call(fn, reps: int = 5, warm: int = 2) -> float:
    """Milliseconds per call of fn() on the current stream (CUDA events)."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_group(group: dict, reps: int = 5, split: bool = False) -> tuple[dict, dict]:
    """Best tuning of one group (dict with step, y, k, dt, sol, delta: a
    MultiNetworkBatch group or a uniform Ros2Step batch) -> (tuning,
    {candidate label: ms})."""
    step = group["step"]
    net = step.net
    timings, best, best_ms = {}, None, float("inf")
    for cand in candidates(net.ni, split):
        set_tuning(net, cand)
        ms = time_call(lambda: step(group["y"], group["k"], group["dt"], out=(group["sol"], group["delta"])), reps)
        timings[json.dumps(cand, sort_keys=True)] = ms
        if ms < best_ms:
            best, best_ms = cand, ms
    set_tuning(net, best)
    return best, timings


def tune_batch(batch, cache_path: str | None = None, reps: int = 5) -> dict:
    """Tune every group of a MultiNetworkBatch (before capture); returns
    {group key: {"tuning": ..., "ms": ..., "candidates": ...}} and, with
    cache_path, merges it into that JSON file."""
    out = {}
    for g in batch.groups:
        best, timings = tune_group(g, reps)
        key = group_key(g["step"].net, g["step"].batch, g["step"].layers)
        out[key] = {"tuning": best, "ms": min(timings.values()), "candidates": timings}
    if cache_path:
        cache = load_cache(cache_path)
        cache.update(out)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    return out


def load_cache(path: str | None) -> dict:
    if not path or not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def apply_cache(batch, cache: dict) -> int:
    """Apply cached tunings to the groups of a MultiNetworkBatch; returns how
    many groups found an entry."""
    hits = 0
    for g in batch.groups:
        key = group_key(g["step"].net, g["step"].batch, g["step"].layers)
        if key in cache:
            set_tuning(g["step"].net, cache[key]["tuning"])
            hits += 1
    return hits
