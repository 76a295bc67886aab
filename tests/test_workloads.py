"""The seeded workload generators: deterministic bytes, expected sizes and shapes."""
from __future__ import annotations

import hashlib
import math

import numpy as np

from quarry import workloads as w


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def test_deterministic_math_is_accurate():
    L = w._lib()
    for x in np.linspace(-300, 300, 2001):
        assert abs(L.qs_det_sin(x) - math.sin(x)) < 1e-14
        assert abs(L.qs_det_cos(x) - math.cos(x)) < 1e-14
    for x in np.geomspace(1e-9, 1e9, 501):
        assert abs(L.qs_det_log(x) - math.log(x)) < 1e-13 * max(1.0, abs(math.log(x)))
    for x in np.linspace(-20, 20, 401):
        assert abs(L.qs_det_exp(x) - math.exp(x)) < 1e-14 * math.exp(x)


def test_terrain_shapes_and_repeatability():
    t = w.terrain(256, 1)
    assert t.shape == (131072, 9)
    assert _sha(t) == _sha(w.terrain(256, 1))
    assert t[:, [0, 3, 6]].min() == 0 and t[:, [0, 3, 6]].max() == 256
    cfg = w.terrain_config(256, 1000, 100, 1)
    assert np.all(cfg.rays[:, 2] == 100) and np.all(cfg.rays[:, 5] == -1)


def test_city_config():
    tris, top = w.city(131072, 1)
    assert tris.shape == (1310720, 9)
    assert top > 50
    z = tris[:, [2, 5, 8]]
    assert z.min() == 0.0
    cfg = w.city_config(2000, 5000, 300, 1)
    d = cfg.rays[:, 3:6]
    assert np.all(d[:, 2] < 0) and np.allclose(np.linalg.norm(d, axis=1), 1, atol=1e-5)


def test_clouds():
    s = w.point_cloud("sphere", 20000, 1)
    r = np.linalg.norm(s, axis=1)
    assert abs(r.mean() - 50) < 0.05 and 0.4 < r.std() < 0.6
    v = w.point_cloud("volume", 20000, 1)
    assert v.min() >= 0 and v.max() <= 100
    moved, ids = w.coherent_motion(v, 0.01, 0.05, 1)
    assert len(ids) == 200 and np.all(np.diff(ids) > 0)
    assert np.count_nonzero(np.any(moved != v, axis=1)) <= 200
    g = w.gaussians(5000, 0.05, 1.0, 1)
    assert np.all(g[:, 7:10] >= 0.0499) and np.all(g[:, 7:10] <= 1.0001)
    assert np.allclose(np.linalg.norm(g[:, 3:7], axis=1), 1, atol=1e-5)


def test_standalone_generators_match_the_engine_library():
    """bench.py's CPU arm makes its inputs from oracle/_build/libqscenes.so (scenes.c built on
    its own) so it never loads the engine; the bytes must equal the engine library's."""
    import oracle

    alone = oracle.standalone_workloads()
    a, b = alone.city_config(2048, 5000, 300, 1), w.city_config(2048, 5000, 300, 1)
    assert np.array_equal(a.tris, b.tris) and np.array_equal(a.rays, b.rays)
    assert np.array_equal(a.queries, b.queries) and a.top == b.top
    a, b = alone.terrain_config(40, 5000, 300, 1), w.terrain_config(40, 5000, 300, 1)
    assert np.array_equal(a.tris, b.tris) and np.array_equal(a.rays, b.rays)
    assert np.array_equal(a.queries, b.queries)
    assert np.array_equal(alone.gaussians(500, 0.05, 1.0, 3), w.gaussians(500, 0.05, 1.0, 3))
    assert np.array_equal(alone.point_cloud("surface", 1000, 2), w.point_cloud("surface", 1000, 2))
