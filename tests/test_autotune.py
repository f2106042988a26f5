"""The autotuner's host side (no GPU): the candidate schedules and the JSON cache."""

import json

from mit_jax_b200 import autotune


def test_candidates_cover_grid_sizes_and_deals():
    c = autotune.candidates(148)
    assert len(c) == 14
    assert {d["unit_deal"] for d in c} == {0, 1}
    assert {d["ctas_per_sm"] for d in c} == {1, 2}
    assert {d["stages"] for d in c} == {2, 3, 4}
    assert {d["grid_ctas"] for d in c if d["ctas_per_sm"] == 2} == {296, 222, 148}
    assert all(set(d) == {"grid_ctas", "ctas_per_sm", "unit_deal", "stages"} and d["grid_ctas"] >= 1 for d in c)
    assert len({json.dumps(d, sort_keys=True) for d in c}) == len(c)


def test_cache_file_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("MIT_JAX_B200_TUNE_CACHE", str(path))
    monkeypatch.setattr(autotune, "_CACHE", {})
    monkeypatch.setattr(autotune, "_LOADED", set())
    sched = {"grid_ctas": 222, "ctas_per_sm": 2, "unit_deal": 1, "stages": 2}
    autotune._CACHE["k"] = sched
    autotune._save(str(path))
    assert json.loads(path.read_text()) == {"k": sched}
    # a fresh process: nothing in memory, the file is read once
    monkeypatch.setattr(autotune, "_CACHE", {})
    monkeypatch.setattr(autotune, "_LOADED", set())
    assert autotune.cached("k") == sched
    assert autotune.cached("other") is None
    # malformed entries are ignored
    path.write_text(json.dumps({"bad": {"grid_ctas": 1}}))
    monkeypatch.setattr(autotune, "_CACHE", {})
    monkeypatch.setattr(autotune, "_LOADED", set())
    assert autotune.cached("bad") is None
