"""Autotuner host logic (CPU): the candidate shapes per species count, the
cache file round trip and group keys. The timing itself runs on the GPU
(tests/test_gpu_ragged.py)."""
import json

from conftest import load_pkg

at = load_pkg("autotune")


def test_candidates_cover_the_compiled_variants():
    c69 = list(at.candidates(69))
    assert len(c69) == 28 and len(list(at.candidates(69, split=True))) == 56
    assert {c["factor_ctas"] for c in c69} == {1, 2}
    assert {c["factor_kernel"] for c in c69} == {1, 2, 3, 4}
    assert all(c["factor_ctas"] == 1 for c in c69 if c["factor_kernel"] == 4)
    assert {c["sweep_stages"] for c in c69} == {2, 3}
    c30 = list(at.candidates(30))
    assert len(c30) == 12 and all(c["factor_ctas"] == 0 for c in c30)


def test_cache_round_trip(tmp_path):
    p = tmp_path / "tune.json"
    assert at.load_cache(str(p)) == {}
    entry = {"k": {"tuning": {"factor_kernel": 1, "factor_ctas": 2, "sweep_stages": 3}, "ms": 1.0, "candidates": {}}}
    p.write_text(json.dumps(entry))
    assert at.load_cache(str(p)) == entry
    assert at.VbTuning(1, 2, 3, 2, 2, 0).sweep_stages == 3
