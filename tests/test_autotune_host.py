"""Autotuner host logic on CPU: the JSON cache, cache keys and the candidate search."""

from __future__ import annotations

import numpy as np

from warp_vp_solver_b200.autotune import TuneCache, ensemble_candidates, plan_candidates, search, signature


def test_cache_round_trip(tmp_path):
    c = TuneCache(str(tmp_path / "sub" / "tune.json"))
    assert c.get("k") is None
    c.put("k", {"config": {"stage_rows": 8}, "ms": 1.5})
    c.put("k2", {"config": {"cluster_size": 4}, "ms": 0.5})
    assert c.get("k")["config"] == {"stage_rows": 8}
    assert TuneCache(c.path).get("k2")["ms"] == 0.5


def test_signature_is_stable_and_distinguishes_shapes():
    a = signature("plan", nx=64, nv=256, dtype="f32")
    assert a == signature("plan", dtype="f32", nv=256, nx=64)
    assert a != signature("plan", nx=64, nv=512, dtype="f32")
    s1 = signature("ensemble", shapes=np.array([[64, 128], [128, 256]]))
    s2 = signature("ensemble", shapes=np.array([[64, 128], [128, 512]]))
    assert s1 != s2


def test_search_picks_fastest_usable_candidate():
    times = {1: 3.0, 2: 1.0, 3: 0.5, 4: 2.0}
    state = {}

    def apply(c):
        if c["x"] == 3:
            return False   # not usable
        state["x"] = c["x"]
        return True

    best, ms, tried = search([{"x": k} for k in times], apply, lambda: times[state["x"]], repeats=2)
    assert best == {"x": 2} and ms == 1.0
    assert [t[0]["x"] for t in tried] == [1, 2, 4]


def test_candidate_sets():
    c = plan_candidates({"cluster_size": 8})
    assert {"cluster_size": 16, "persist_rows": 0, "strip_rows": 0} in c and any(x.get("stage_rows") == 16 for x in c)
    c = plan_candidates({"cluster_size": 0})
    assert not any("stage_rows" not in x and x["cluster_size"] > 0 for x in c)
    assert {"cluster_size": 0, "persist_rows": 16, "strip_rows": 0} in c
    assert {"cluster_size": 0, "persist_rows": 0, "strip_rows": 16} in c
    # every candidate names both loop paths, and at most one of them is on
    assert all("persist_rows" in x and "strip_rows" in x for x in c)
    assert all(x["persist_rows"] == 0 or x["strip_rows"] == 0 for x in c)
    assert all(x["persist_rows"] == 0 and x["strip_rows"] == 0 for x in c if "stage_rows" in x or x["cluster_size"] > 0)
    e = ensemble_candidates({})
    assert all(x["rows_per_tile"] in (1, 2, 4, 8) for x in e) and len(e) > 10
