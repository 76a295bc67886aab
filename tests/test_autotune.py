"""The autotuner's search, persistence and result check, with a fake timer (no GPU)."""
from __future__ import annotations

import json

import pytest

from quarry import autotune


def fake_timer(costs):
    calls = []

    def timer(run, params, repeats):
        calls.append(dict(params))
        run(params)
        return costs(params)

    return timer, calls


SPACE = {"a": [0, 1, 2, 3], "b": ["x", "y", "z"], "c": [1, 2]}


def separable(p):
    return 10.0 + abs(p["a"] - 2) * 3 + {"x": 2.0, "y": 0.0, "z": 5.0}[p["b"]] + (p["c"] - 1)


def test_coordinate_descent_finds_separable_optimum(tmp_path):
    timer, calls = fake_timer(separable)
    tu = autotune.Autotuner(tmp_path / "t.json", timer=timer, device="dev")
    res = tu.search("w", SPACE, run=lambda p: None)
    assert res.params == {"a": 2, "b": "y", "c": 1}
    assert res.ms == 10.0 and not res.cached
    # each point is measured once
    assert len(calls) == len({json.dumps(c, sort_keys=True) for c in calls})
    assert len(calls) < 4 * 3 * 2


def test_choices_persist_and_are_reused(tmp_path):
    timer, calls = fake_timer(separable)
    tu = autotune.Autotuner(tmp_path / "t.json", timer=timer, device="dev")
    tu.search("w", SPACE, run=lambda p: None)
    tu.save()
    timer2, calls2 = fake_timer(lambda p: 1.0)
    tu2 = autotune.Autotuner(tmp_path / "t.json", timer=timer2, device="dev")
    res = tu2.search("w", SPACE, run=lambda p: None)
    assert res.cached and res.params == {"a": 2, "b": "y", "c": 1} and not calls2
    assert tu2.lookup("w") == res.params
    # another device or workload key measures again
    tu3 = autotune.Autotuner(tmp_path / "t.json", timer=timer2, device="other")
    assert tu3.lookup("w") is None
    assert not tu3.search("w", SPACE, run=lambda p: None).cached


def test_corrupt_or_old_cache_is_ignored(tmp_path):
    p = tmp_path / "t.json"
    p.write_text("{not json")
    assert autotune.Autotuner(p, timer=fake_timer(separable)[0], device="d").cache == {}
    p.write_text(json.dumps({"version": 0, "entries": {"d|w": {"params": {}, "ms": 1}}}))
    assert autotune.Autotuner(p, timer=fake_timer(separable)[0], device="d").cache == {}


def test_candidate_that_changes_results_is_an_error(tmp_path):
    timer, _ = fake_timer(separable)
    tu = autotune.Autotuner(tmp_path / "t.json", timer=timer, device="dev")
    state = {}

    def run(p):
        state["last"] = p

    def fp(p):
        return 7 if state["last"]["b"] != "z" else 8

    with pytest.raises(autotune.FingerprintMismatch):
        tu.search("w", SPACE, run=run, fingerprint=fp)


def test_invalid_points_are_skipped(tmp_path):
    timer, calls = fake_timer(lambda p: 1.0 if p["b"] == "z" else 5.0)
    tu = autotune.Autotuner(tmp_path / "t.json", timer=timer, device="dev")
    res = tu.search("w", SPACE, run=lambda p: None, valid=lambda p: p["b"] != "z")
    assert res.params["b"] != "z"
    assert all(c["b"] != "z" for c in calls)


def test_batch_split_validity():
    ok = autotune.batch_valid("rays")
    assert ok({"flags": 1, "split": 0}) and not ok({"flags": 1, "split": 1})
    ok = autotune.batch_valid("knn")
    assert ok({"flags": 1, "split": 1}) and not ok({"flags": 5, "split": 1})
    assert autotune.batch_launch({**autotune.BATCH_START, "split": 1})["split"] == 1


def test_engine_spaces_are_consistent():
    assert all(autotune.BATCH_START[k] in v for k, v in autotune.BATCH_SPACE.items())
    assert set(autotune.batch_launch(autotune.BATCH_START)) == {
        "block", "blocks_per_sm", "short_stack", "chunks_per_fetch", "split"}
    assert autotune.ray_valid({"layout": "wide", "schedule": "plain"})
    assert not autotune.ray_valid({"layout": "wide", "schedule": "dyn"})
    # the shared-memory short stack stays within 48 KB for every block size
    for b in autotune.BATCH_SPACE["block"]:
        for s in autotune.BATCH_SPACE["short_stack"]:
            assert b * s * 8 <= 48 * 1024


def test_shipped_choices_are_a_fallback(tmp_path):
    shipped = tmp_path / "shipped.json"
    shipped.write_text(json.dumps({"version": autotune.VERSION, "entries": {
        "dev|w": {"params": {"a": 3, "b": "x", "c": 2}, "ms": 2.0}}}))
    timer, calls = fake_timer(separable)
    tu = autotune.Autotuner(tmp_path / "cache.json", timer=timer, device="dev", shipped=shipped)
    res = tu.search("w", SPACE, run=lambda p: None)
    assert res.cached and res.source == "shipped" and res.params["a"] == 3 and not calls
    # force measures and the measured choice then shadows the shipped one
    res = tu.search("w", SPACE, run=lambda p: None, force=True)
    assert not res.cached and res.params == {"a": 2, "b": "y", "c": 1}
    assert tu.search("w", SPACE, run=lambda p: None).source == "cache"


def test_shipped_b200_table_is_valid():
    data = json.loads(autotune.SHIPPED.read_text())
    assert data["version"] == autotune.VERSION and data["entries"]
    for key, e in data["entries"].items():
        p = e["params"]
        if "|batch-step:" in key:
            assert p["builder"] in ("lbvh", "sah8", "sah16", "sah32")
            continue
        assert "|batch:" in key
        assert all(p.get(k, autotune.BATCH_START[k]) in v
                   for k, v in autotune.BATCH_SPACE.items()), (key, p)
