"""The oracle (oracle/quarry_oracle.c) pinned against quarry's own CPU reference.

oracle/_ref/libquarry_ref.so is compiled from the reference's src/core and src/cpu sources
by oracle/Makefile.  These tests run both on the same seeded inputs and require identical
bits: ray results, closest / kNN / radius results and the FNV-1a fingerprints folded the
reference's way (src/core/fingerprint.h).  They also run the reference's own self test.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from quarry import workloads

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference sources not present on this machine")


def _random_rays(lo, hi, n, seed):
    rng = np.random.default_rng(seed)
    c = (lo + hi) / 2
    ext = hi - lo
    rad = 1.6 * float(np.linalg.norm(ext))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = c + d * rad
    tgt = c + (rng.random((n, 3)) * 2 - 1) * ext * 0.9
    dirs = tgt - o
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = o
    rays[:, 3:6] = dirs
    rays[:, 6] = 1e-6
    rays[:, 7] = rad * 4
    return rays


@needs_ref
def test_reference_selftest_passes():
    assert oracle.Reference().selftest()


@needs_ref
@pytest.mark.parametrize("scene", ["terrain", "mixed", "city"])
def test_rays_match_reference(scene):
    if scene == "terrain":
        tris = workloads.terrain(40, 2)
    elif scene == "mixed":
        tris = workloads.demo_mesh_tris(2, 20, 1500, 7, 0)
    else:
        tris, _ = workloads.city(400, 3)
    lo, hi = workloads.bounds_of(tris)
    R = oracle.Reference()
    bv = oracle.LBVH("tri", tris)
    for rays in (workloads.down_rays(4000, float(lo[0]), float(hi[0]), float(lo[1]),
                                     float(hi[1]), float(hi[2]) + 3, 4),
                 _random_rays(lo, hi, 4000, 5),
                 workloads.cosine_rays(4000, float(lo[0]), float(hi[0]), float(lo[1]),
                                       float(hi[1]), float(hi[2]) + 3, 6)):
        got = bv.raycast(rays)
        want, _, _ = R.raycast(tris, rays)
        assert np.array_equal(got, want)
        assert oracle.ray_hash(got) == R.ray_hash(want)
        # brute force agrees too (both implementations)
        assert np.array_equal(oracle.raycast_brute(tris, rays[:300]), want[:300])
        assert np.array_equal(R.raycast_brute(tris, rays[:300]), want[:300])


def _kind_items(kind):
    if kind == "tri":
        return workloads.demo_mesh_tris(2, 16, 800, 3, 0)
    if kind == "point":
        return workloads.point_cloud("sphere", 15000, 2)
    return workloads.gaussians(3000, 0.05, 1.0, 2)


@needs_ref
@pytest.mark.parametrize("kind", ["tri", "point", "gauss"])
def test_queries_match_reference(kind):
    items = _kind_items(kind)
    if kind == "tri":
        lo, hi = workloads.bounds_of(items)
    else:
        lo, hi = items[:, :3].min(0), items[:, :3].max(0)
    q = workloads.uniform_points(1500, lo - 2, hi + 2, 9, 21)
    R = oracle.Reference()
    bv = oracle.LBVH(kind, items)
    got = bv.closest(q)
    want, _, _ = R.closest(kind, items, q)
    assert np.array_equal(got, want)
    assert oracle.closest_hash(got) == R.closest_hash(want)
    assert np.array_equal(oracle.closest_brute(kind, items, q[:200]), want[:200])
    for k in (1, 8, 32):
        got = bv.knn(q, k)
        want, _, _ = R.knn(kind, items, q, k)
        assert np.array_equal(got, want)
        off, keys = oracle.knn_to_csr(got)
        assert oracle.knn_hash(got) == R.list_hash(off, keys)
    r = {"tri": 2.0, "point": 3.0, "gauss": 1.5}[kind]
    off, keys = bv.radius(q, r)
    woff, wkeys, _ = R.radius(kind, items, q, r)
    assert np.array_equal(off, woff) and np.array_equal(keys, wkeys)
    assert oracle.radius_hash(off, keys) == R.list_hash(woff, wkeys)


@needs_ref
def test_leaf_tests_match_reference_on_edge_cases():
    """Degenerate triangles, zero directions, axis-parallel rays, points on edges."""
    R = oracle.Reference().leaf()
    import ctypes

    rng = np.random.default_rng(17)
    tris = rng.normal(size=(400, 9)).astype(np.float32)
    tris[::7, 6:9] = tris[::7, 0:3]  # collapsed corner
    tris[::11, 3:6] = tris[::11, 0:3] * 2 - tris[::11, 6:9]  # collinear
    pts = rng.normal(size=(400, 3)).astype(np.float32) * 2
    pts[::5] = tris[::5, 0:3]  # on a vertex
    rays = np.zeros((400, 8), np.float32)
    rays[:, :3] = rng.normal(size=(400, 3)) * 3
    rays[:, 3:6] = rng.normal(size=(400, 3))
    rays[::4, 3:5] = 0.0  # axis-parallel
    rays[::13, 3:6] = 0.0  # zero direction
    rays[:, 6] = 1e-6
    rays[:, 7] = np.inf
    P = ctypes.c_void_p
    for i in range(400):
        t1, t2 = ctypes.c_float(0), ctypes.c_float(0)
        a = oracle.lib().qo_intersect_triangle(rays[i].ctypes.data_as(P), tris[i].ctypes.data_as(P), ctypes.byref(t1))
        b = R.qr_intersect_triangle(rays[i].ctypes.data_as(P), tris[i].ctypes.data_as(P), ctypes.byref(t2))
        assert a == b and (not a or np.float32(t1.value).tobytes() == np.float32(t2.value).tobytes())
        d1 = oracle.lib().qo_closest_point_dist2(pts[i].ctypes.data_as(P), tris[i].ctypes.data_as(P))
        d2 = R.qr_closest_point_dist2(pts[i].ctypes.data_as(P), tris[i].ctypes.data_as(P))
        assert np.float32(d1).tobytes() == np.float32(d2).tobytes()
    g = workloads.gaussians(400, 0.01, 3.0, 5)
    g[::9, 7:10] = g[::9, 7:8]  # spheres
    g[::10, 3:7] = 0.0  # zero quaternion
    for i in range(400):
        d1 = oracle.lib().qo_gaussian_dist2(pts[i].ctypes.data_as(P), g[i].ctypes.data_as(P))
        d2 = R.qr_gaussian_dist2(pts[i].ctypes.data_as(P), g[i].ctypes.data_as(P))
        assert np.float32(d1).tobytes() == np.float32(d2).tobytes()
        b1 = oracle.prim_bounds("gauss", g[i])
        b2 = np.zeros(6, np.float32)
        R.qr_gaussian_bounds(g[i].ctypes.data_as(P), b2.ctypes.data_as(P))
        assert b1.tobytes() == b2.tobytes()
