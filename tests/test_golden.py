"""The oracle against golden vectors: known answers of quarry's self test
(src/cpu/selftest.cpp:28-52, 100-123) and fixtures recorded from quarry's own CPU reference
(tests/golden/*.npz, made by tests/golden/make_golden.py).  Runs on the CPU."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
TRI = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32)


def ray(o, d):
    return np.array([*o, *d, 1e-6, np.inf], np.float32)


def test_known_answer_triangle():
    ok, t = oracle.intersect_triangle(ray((0.25, 0.25, 1.0), (0, 0, -1)), TRI)
    assert ok and abs(t - 1.0) < 1e-5
    assert not oracle.intersect_triangle(ray((2, 2, 1), (0, 0, -1)), TRI)[0]
    assert not oracle.intersect_triangle(ray((0, 0, 1), (1, 0, 0)), TRI)[0]
    assert not oracle.intersect_triangle(ray((0.25, 0.25, 1), (0, 0, 1)), TRI)[0]
    ok, t = oracle.intersect_triangle(ray((0.25, 0.25, -1), (0, 0, 1)), TRI)
    assert ok and abs(t - 1.0) < 1e-5


@pytest.mark.parametrize("p,d2", [((0.25, 0.25, 1.0), 1.0), ((-1, -1, 0), 2.0), ((2, 0, 0), 1.0),
                                  ((0.5, 0.5, 0), 0.0), ((0.5, -1, 0), 1.0)])
def test_known_answer_closest_point(p, d2):
    assert abs(oracle.prim_dist2("tri", np.array(p, np.float32), TRI) - d2) < 1e-6


def test_known_answer_box_distance():
    import ctypes

    box = np.array([0, 0, 0, 1, 1, 1], np.float32)
    f = oracle.lib().qo_dist2_aabb
    P = ctypes.c_void_p
    for p, want in (((0.5, 0.5, 0.5), 0.0), ((2, 0.5, 0.5), 1.0), ((2, 3, 1), 5.0)):
        q = np.array(p, np.float32)
        assert abs(f(q.ctypes.data_as(P), box.ctypes.data_as(P)) - want) < 1e-6


@pytest.mark.parametrize("name", ["tri", "city", "point", "gauss"])
def test_oracle_matches_golden_fixtures(name):
    g = np.load(GOLDEN / f"{name}.npz")
    kind = "tri" if name in ("tri", "city") else name
    bv = oracle.LBVH(kind, g["items"])
    q = g["queries"]
    assert np.array_equal(bv.closest(q), g["closest"])
    assert np.array_equal(bv.knn(q, 8), g["knn8"])
    off, keys = bv.radius(q, float(g["radius"]))
    assert np.array_equal(off, g["radius_offsets"]) and np.array_equal(keys, g["radius_keys"])
    if "rays" in g:
        assert np.array_equal(bv.raycast(g["rays"]), g["ray_results"])
        assert np.array_equal(oracle.raycast_brute(g["items"], g["rays"]), g["ray_results"])
