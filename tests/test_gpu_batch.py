"""Batched scenes on the GPU: trees bit-identical to single builds, every query result
bit-identical to the oracle, for both schedules, both layouts and several launch shapes."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from quarry import capi, workloads

pytestmark = pytest.mark.gpu

_CFG = None


def small_config():
    global _CFG
    if _CFG is None:
        _CFG = workloads.batch_config(terrains=5, clouds=5, tri_range=(1_000, 20_000),
                                      point_range=(4_000, 40_000), query_range=(200, 3_000), k=16)
    return _CFG


def _batch(cuda, kind, wide=True, schedule=capi.QK_SCHEDULE_BATCHED):
    cfg = small_config()
    scenes = cfg.terrains if kind == "tri" else cfg.clouds
    b = capi.Batch(kind, [s.items for s in scenes], wide=wide)
    b.build(schedule)
    b.sync()
    return b, scenes


def _dev(a):
    return capi.to_device(np.ascontiguousarray(a), np.float32)


@pytest.mark.parametrize("kind", ["tri", "point"])
@pytest.mark.parametrize("schedule", [capi.QK_SCHEDULE_BATCHED, capi.QK_SCHEDULE_LOOP])
def test_batch_trees_equal_single_builds(cuda, kind, schedule):
    b, scenes = _batch(cuda, kind, schedule=schedule)
    for i, sc in enumerate(scenes):
        ref = oracle.LBVH(kind, sc.items)
        v = b.view(i)
        assert v.t.depth == ref.depth
        assert np.array_equal(v.nodes_bytes(), ref.nodes.view(np.uint8)), f"scene {i}"
        assert v.validate() == [0] * 8
        wide, _ = ref.wide()
        assert v.t.wide_count == wide.shape[0] // 4
        got = v.arrays["wide"].cpu().numpy()[: wide.nbytes]
        assert np.array_equal(got, wide.view(np.uint8)), f"scene {i} wide"


def _queries(cfg_scenes, field):
    parts = [getattr(s, field) for s in cfg_scenes]
    counts = np.array([p.shape[0] for p in parts], np.int32)
    return np.concatenate(parts, axis=0), counts


TUNES = [None, {"block": 64, "blocks_per_sm": 8, "short_stack": 0, "chunks_per_fetch": 1},
         {"block": 256, "blocks_per_sm": 2, "short_stack": 16, "chunks_per_fetch": 8}]
SPLIT = {"block": 128, "blocks_per_sm": 6, "short_stack": 0, "chunks_per_fetch": 2, "split": 1}


@pytest.mark.parametrize("flags", [0, capi.QK_ORDER_MORTON, capi.QK_WIDE,
                                   capi.QK_WIDE | capi.QK_ORDER_MORTON])
@pytest.mark.parametrize("schedule", [capi.QK_SCHEDULE_BATCHED, capi.QK_SCHEDULE_LOOP])
def test_batch_rays_match_oracle(cuda, flags, schedule):
    b, scenes = _batch(cuda, "tri")
    rays, counts = _queries(scenes, "rays")
    plan = b.plan(capi.QK_OP_RAY, counts, flags=flags)
    rd = _dev(rays)
    want = np.concatenate([oracle.LBVH("tri", s.items).raycast(s.rays) for s in scenes])
    for tune in (TUNES if schedule == capi.QK_SCHEDULE_BATCHED else [None]):
        out = cuda.zeros(rays.shape[0], dtype=cuda.int64, device="cuda")
        plan.query(rd, out, tune=tune, schedule=schedule)
        assert plan.status()[1] == 0
        assert np.array_equal(out.cpu().numpy().view(np.uint64), want)


@pytest.mark.parametrize("kind", ["tri", "point"])
@pytest.mark.parametrize("flags", [0, capi.QK_ORDER_MORTON | capi.QK_WIDE])
@pytest.mark.parametrize("schedule", [capi.QK_SCHEDULE_BATCHED, capi.QK_SCHEDULE_LOOP])
def test_batch_closest_knn_match_oracle(cuda, kind, flags, schedule):
    b, scenes = _batch(cuda, kind)
    cfg = small_config()
    pts, counts = _queries(scenes, "closest")
    plan = b.plan(capi.QK_OP_CLOSEST, counts, flags=flags)
    out = cuda.zeros((pts.shape[0], 2), dtype=cuda.int32, device="cuda")
    tunes = TUNES + ([SPLIT] if not flags & capi.QK_WIDE else [])
    for tune in (tunes if schedule == capi.QK_SCHEDULE_BATCHED else [None]):
        plan.query(_dev(pts), out, tune=tune, schedule=schedule)
        want = np.concatenate([oracle.LBVH(kind, s.items).closest(s.closest) for s in scenes])
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
    pts, counts = _queries(scenes, "knn")
    plan = b.plan(capi.QK_OP_KNN, counts, flags=flags)
    want = np.concatenate([oracle.LBVH(kind, s.items).knn(s.knn, cfg.k) for s in scenes])
    tunes = [TUNES[2]] + ([SPLIT] if not flags & capi.QK_WIDE else [])
    for tune in (tunes if schedule == capi.QK_SCHEDULE_BATCHED else [None]):
        out = cuda.zeros((pts.shape[0], cfg.k, 2), dtype=cuda.int32, device="cuda")
        plan.query(_dev(pts), out, k=cfg.k, schedule=schedule, tune=tune)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)


@pytest.mark.parametrize("kind", ["tri", "point"])
@pytest.mark.parametrize("flags", [0, capi.QK_ORDER_MORTON | capi.QK_WIDE])
@pytest.mark.parametrize("schedule", [capi.QK_SCHEDULE_BATCHED, capi.QK_SCHEDULE_LOOP])
def test_batch_radius_matches_oracle(cuda, kind, flags, schedule):
    b, scenes = _batch(cuda, kind)
    pts, counts = _queries(scenes, "radius")
    radii = np.array([s.r for s in scenes], np.float32)
    plan = b.plan(capi.QK_OP_RADIUS, counts, params=radii, flags=flags)
    want = [oracle.LBVH(kind, s.items).radius(s.radius, float(s.r)) for s in scenes]
    total = sum(int(w[0][-1]) for w in want)
    keys = cuda.zeros(total + 16, dtype=cuda.int64, device="cuda")
    offsets = cuda.zeros(pts.shape[0] + len(scenes) + 1, dtype=cuda.int32, device="cuda")
    tune = SPLIT if schedule == capi.QK_SCHEDULE_BATCHED and not flags & capi.QK_WIDE else None
    plan.query(_dev(pts), keys, offsets=offsets, capacity=keys.numel(), schedule=schedule,
               tune=tune)
    got_total, ovf = plan.status()
    assert got_total == total and ovf == 0
    off = offsets.cpu().numpy().astype(np.int64)
    k = keys.cpu().numpy().view(np.uint64)
    base = 0
    for i, (wo, wk) in enumerate(want):
        q0, q1 = int(plan.q_off[i]), int(plan.q_off[i + 1])
        if schedule == capi.QK_SCHEDULE_BATCHED:
            so = off[q0:q1 + 1] - off[q0]
            sk = k[off[q0]:off[q1]]
        else:
            so = off[q0 + i:q1 + i + 1]
            sk = k[base:base + int(so[-1])]
            base += int(so[-1])
        assert np.array_equal(so, wo), f"scene {i} offsets"
        assert np.array_equal(sk, wk), f"scene {i} keys"


def test_batch_radius_capacity_guard(cuda):
    b, scenes = _batch(cuda, "point")
    pts, counts = _queries(scenes, "radius")
    radii = np.array([s.r for s in scenes], np.float32)
    plan = b.plan(capi.QK_OP_RADIUS, counts, params=radii)
    keys = cuda.full((8,), -1, dtype=cuda.int64, device="cuda")
    offsets = cuda.zeros(pts.shape[0] + len(scenes) + 1, dtype=cuda.int32, device="cuda")
    plan.query(_dev(pts), keys, offsets=offsets, capacity=4)
    with pytest.raises(capi.QkError):
        plan.status()
    # nothing was written past the capacity
    assert (keys.cpu().numpy()[4:] == -1).all()


def test_batch_graph_capture_replays(cuda):
    """Build + rays captured in one CUDA graph give the same bits on every replay."""
    cfg = small_config()
    b = capi.Batch("tri", [s.items for s in cfg.terrains], wide=False)
    b.build()
    b.sync()
    rays, counts = _queries(cfg.terrains, "rays")
    plan = b.plan(capi.QK_OP_RAY, counts, flags=capi.QK_ORDER_MORTON)
    rd = _dev(rays)
    out = cuda.zeros(rays.shape[0], dtype=cuda.int64, device="cuda")
    s = cuda.cuda.Stream()
    s.wait_stream(cuda.cuda.current_stream())
    g = cuda.cuda.CUDAGraph()
    with cuda.cuda.stream(s):
        with cuda.cuda.graph(g, stream=s):
            b.build()
            plan.query(rd, out)
    want = np.concatenate([oracle.LBVH("tri", sc.items).raycast(sc.rays) for sc in cfg.terrains])
    for _ in range(3):
        out.zero_()
        g.replay()
        cuda.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint64), want)
    b.sync()


@pytest.mark.parametrize("bins", [8, 32])
def test_batch_sah_trees_give_oracle_results(cuda, bins):
    """Per-scene SAH builds into the batch arena: valid trees whose batched query results
    equal the oracle's (results do not depend on the tree)."""
    cfg = small_config()
    b = capi.Batch("tri", [s.items for s in cfg.terrains], wide=True)
    b.build_sah(bins)
    b.sync()
    for i in range(len(cfg.terrains)):
        assert b.view(i).validate() == [0] * 8
    rays, counts = _queries(cfg.terrains, "rays")
    for flags in (0, capi.QK_WIDE | capi.QK_ORDER_MORTON):
        plan = b.plan(capi.QK_OP_RAY, counts, flags=flags)
        out = cuda.zeros(rays.shape[0], dtype=cuda.int64, device="cuda")
        plan.query(_dev(rays), out)
        want = np.concatenate([oracle.LBVH("tri", s.items).raycast(s.rays) for s in cfg.terrains])
        assert np.array_equal(out.cpu().numpy().view(np.uint64), want)
