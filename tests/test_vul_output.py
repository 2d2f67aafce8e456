"""``.vul`` output (reference `legacy_io.py:429-790`): the pickle written for
one atmosphere of a batched loop carry holds the three top-level dicts with
the keys, types and shapes the reference writer publishes and its comparison
tool reads (species, nr, y_ini, y, ymix, t, dt, longdy, atom_loss per atom,
the k dict by row, the counters). Host only; no GPU."""
import pickle

import numpy as np

from conftest import load_pkg

lio = load_pkg("legacy_io")


def fake_carry(B=2, nz=5, ni=4, nr=6, n_atoms=2, seed=0):
    rng = np.random.default_rng(seed)
    snap = {"y": rng.uniform(1.0, 2.0, (B, nz, ni)), "ymix": rng.uniform(0.1, 0.3, (B, nz, ni)),
            "y_prev": rng.uniform(1.0, 2.0, (B, nz, ni)), "dt": rng.uniform(1e-3, 1.0, B), "t": rng.uniform(1, 10, B),
            "delta": rng.uniform(0, 1, B), "small_y": np.zeros(B), "nega_y": np.zeros(B),
            "atom_loss": rng.normal(0, 1e-6, (B, n_atoms)), "atom_loss_prev": np.zeros((B, n_atoms)),
            "accept_count": np.array([17, 23]), "retry_count": np.zeros(B, int), "nega_count": np.array([1, 2]),
            "loss_count": np.array([0, 3]), "delta_count": np.array([4, 5]), "rtol": np.full(B, 0.2),
            "loss_criteria": np.full(B, 1e-3)}
    conv = np.zeros(B, [("longdy", "<f8"), ("longdydt", "<f8"), ("longdy_seen_min", "<f8"), ("aflux_change", "<f8"),
                        ("count_since_new_min", "<i4"), ("done", "<i4"), ("update_photo_frq", "<i4"),
                        ("is_final_photo_frq", "<i4")])
    conv["longdy"], conv["longdydt"], conv["done"], conv["is_final_photo_frq"] = [0.3, 0.01], [1e-3, 1e-5], [0, 1], [0, 1]
    k = rng.uniform(0, 1, (B, nr + 1, nz))
    compo = rng.integers(0, 3, (ni, n_atoms)).astype(float)
    atm = {"Tco": rng.uniform(500, 2000, (B, nz)), "Kzz": rng.uniform(1e7, 1e9, (B, nz - 1)), "ms": np.ones((B, ni)),
           "use_vm_mol": False}
    return snap, conv, k, compo, atm


def test_vul_round_trip(tmp_path):
    snap, conv, k, compo, atm = fake_carry()
    y_ini = snap["y"] * 0.9
    species = ["A", "B", "C", "D"]
    for b in range(2):
        path = lio.write_vul(tmp_path / f"atm{b}.vul", species, k, snap, b=b, y_ini=y_ini, compo=compo,
                             atom_order=["H", "O"], atom_ini=np.einsum("bzi,ia->ba", y_ini, compo), conv=conv,
                             atm=atm, Rf={1: "A + B -> C", 3: "C -> D"})
        with open(path, "rb") as f:
            d = pickle.load(f)
        assert set(d) == {"variable", "atm", "parameter"}
        v, a, p = d["variable"], d["atm"], d["parameter"]
        assert v["species"] == species and v["nr"] == 6
        np.testing.assert_array_equal(v["y_ini"], y_ini[b])
        np.testing.assert_array_equal(v["y"], snap["y"][b])
        np.testing.assert_array_equal(v["ymix"], snap["ymix"][b])
        assert v["t"] == snap["t"][b] and v["dt"] == snap["dt"][b]
        assert v["longdy"] == conv["longdy"][b] and v["longdydt"] == conv["longdydt"][b]
        assert sorted(v["k"]) == list(range(1, 7)) and np.array_equal(v["k"][3], k[b, 3])
        assert set(v["atom_loss"]) == {"H", "O"} and v["atom_loss"]["O"] == snap["atom_loss"][b, 1]
        np.testing.assert_allclose([v["atom_sum"]["H"]], [np.einsum("zi,i->", snap["y"][b], compo[:, 0])])
        assert all(isinstance(x, float) for x in v["atom_loss"].values())
        assert v["Rf"][1] == "A + B -> C"
        np.testing.assert_array_equal(a["Tco"], atm["Tco"][b])
        assert a["use_vm_mol"] is False
        assert p["count"] == snap["accept_count"][b] and p["delta_count"] == snap["delta_count"][b]
        assert p["end_case"] == int(conv["done"][b]) and p["switch_final_photo_frq"] == bool(conv["is_final_photo_frq"][b])
        assert p["where_varies_most"].shape == snap["y"][b].shape


def _reference_dir():
    """The reference checkout: $VULCAN_REFERENCE, else a `reference` directory
    beside this repository (None when neither exists)."""
    import os
    from conftest import ROOT
    for cand in (os.environ.get("VULCAN_REFERENCE"), os.path.join(os.path.dirname(ROOT), "reference")):
        if cand and os.path.exists(os.path.join(cand, "tests", "compare_vul.py")):
            return cand
    return None


def test_vul_read_by_reference_comparison_tool(tmp_path, capsys):
    """The reference's own reader and comparison tool (`tests/compare_vul.py`:
    load_vul, the static invariants, time alignment, atom-loss table and
    per-species log10 ymix metrics) run on files from write_vul: a file
    against itself passes with bit-exact invariants, and two atmospheres of
    the same network and initial state are compared species by species."""
    import importlib.util
    import pytest
    ref = _reference_dir()
    if ref is None:
        pytest.skip("reference checkout not available")
    spec = importlib.util.spec_from_file_location("ref_compare_vul", f"{ref}/tests/compare_vul.py")
    cv = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cv)
    snap, conv, k, compo, atm = fake_carry()
    y_ini = snap["y"][0] * 0.9
    y_ini_b = np.stack([y_ini, y_ini])
    species = ["A", "B", "C", "D"]
    snap["t"][1] = snap["t"][0] * 1.01
    paths = [lio.write_vul(tmp_path / f"atm{b}.vul", species, k, snap, b=b, y_ini=y_ini_b, compo=compo,
                           atom_order=["H", "O"], atom_ini=np.einsum("bzi,ia->ba", y_ini_b, compo), conv=conv,
                           atm=atm) for b in range(2)]
    d = cv.load_vul(paths[0])
    ok, msgs = cv._check_static_invariants(d["variable"], d["variable"])
    assert ok and any("bit-exact" in m for m in msgs), msgs
    assert cv.main([str(paths[0]), str(paths[0])]) == 0
    out = capsys.readouterr().out
    assert "species list: identical (4 species)" in out and "y_ini       : bit-exact" in out
    rc = cv.main([str(paths[0]), str(paths[1]), "--floor", "1e-3"])
    out = capsys.readouterr().out
    assert rc in (0, 1) and "Per-species" in out and "H" in out, out
