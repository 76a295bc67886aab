"""The `quarry` Python module (the reference's module surface) on the GPU.

Follows the checks of quarry's python/test_quarry.py: brute-force agreement for triangles
(with the reference's tolerances where it uses them) and bit-exact agreement for points,
bitwise invariance under order="morton", builder="sah", wide=True and refit / topology
edits against a fresh build, and ValueError on bad input.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import quarry

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mesh(cuda):
    v, i = quarry.demo_mesh("terrain", grid=32)
    return v, i


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_scene_basics_and_queries(mesh):
    assert quarry.describe()
    v, i = mesh
    assert v.shape == (2048 * 3, 3) and i.shape == (2048, 3)
    scene = quarry.Scene(v, i)
    assert scene.triangle_count == 2048 and scene.node_count == 4095
    assert scene.validate() == ""
    assert scene.build_ms > 0
    lo, hi = np.array(scene.bounds["min"]), np.array(scene.bounds["max"])
    rng = np.random.default_rng(7)
    pts = (lo + (hi - lo) * rng.random((300, 3))).astype(np.float32)
    tris = v[i].astype(np.float32)
    d2, tri = scene.closest(pts)
    want = oracle.closest_brute("tri", tris.reshape(-1, 9), pts)
    assert np.array_equal(_bits(d2), want[:, 0]) and np.array_equal(tri, want[:, 1].view(np.int32))
    assert scene.last_query_ms > 0
    kd, kid = scene.knn(pts, 4)
    wk = oracle.knn_brute("tri", tris.reshape(-1, 9), pts, 4)
    assert np.array_equal(_bits(kd), wk[..., 0]) and np.array_equal(kid, wk[..., 1].view(np.int32))
    assert np.array_equal(kid[:, 0], tri)
    radius = 0.3 * float(np.max(hi - lo))
    off, rd2, rid = scene.radius(pts, radius)
    assert off.shape == (301,) and off[0] == 0 and off[-1] == len(rid)
    for j in range(len(pts)):
        seg = rd2[off[j]:off[j + 1]]
        assert np.all(np.diff(seg) >= 0)
    ref = oracle.LBVH("tri", tris.reshape(-1, 9))
    woff, wkeys = ref.radius(pts, radius)
    assert np.array_equal(off, woff)
    assert np.array_equal(_bits(rd2), (wkeys >> np.uint64(32)).astype(np.uint32))
    # order / builder / wide invariance, bit for bit
    for kw in ({"order": "morton"}, {"wide": True}, {"order": "morton", "wide": True},
               {"order": "coherent"}, {"order": "coherent", "wide": True}):
        m_d2, m_tri = scene.closest(pts, **kw)
        assert np.array_equal(_bits(m_d2), _bits(d2)) and np.array_equal(m_tri, tri)
        m_kd, m_kid = scene.knn(pts, 4, **kw)
        assert np.array_equal(_bits(m_kd), _bits(kd)) and np.array_equal(m_kid, kid)
        m_off, m_rd2, m_rid = scene.radius(pts, radius, **kw)
        assert np.array_equal(m_off, off) and np.array_equal(m_rid, rid)
    sah = quarry.Scene(v, i, builder="sah")
    assert sah.validate() == "" and sah.node_count == 4095
    s_d2, s_tri = sah.closest(pts)
    assert np.array_equal(_bits(s_d2), _bits(d2)) and np.array_equal(s_tri, tri)
    assert "sah_bin_ms" in sah.build_stats
    # rays
    origins = (lo + (hi - lo) * rng.random((200, 3))).astype(np.float32)
    origins[:, 1] = hi[1] + 1.0
    dirs = np.tile(np.array([0.0, -1.0, 0.0], np.float32), (200, 1))
    hit, t = scene.raycast(origins, dirs)
    rays = np.zeros((200, 8), np.float32)
    rays[:, :3], rays[:, 3:6], rays[:, 6], rays[:, 7] = origins, dirs, 1e-6, np.inf
    want = oracle.raycast_brute(tris.reshape(-1, 9), rays)
    assert np.array_equal(hit, (want >> np.uint64(32)) != 0)
    assert np.array_equal(_bits(t[hit]), (want[hit] & np.uint64(0xFFFFFFFF)).astype(np.uint32))
    assert np.all(np.isinf(t[~hit]))
    for kw in ({"order": "morton"}, {"order": "direction"}, {"wide": True},
               {"order": "coherent"}, {"order": "coherent", "wide": True}):
        h2, t2 = scene.raycast(origins, dirs, **kw)
        assert np.array_equal(h2, hit) and np.array_equal(_bits(t2), _bits(t))


def test_scene_refit_and_topology(mesh):
    v, i = mesh
    scene = quarry.Scene(v, i)
    lifted = v.copy()
    lifted[:, 1] += 0.1
    scene.update_vertices(lifted)
    assert scene.validate() == "" and scene.refit_stats["updated"] == 2048
    assert scene.refit_ms > 0
    rng = np.random.default_rng(3)
    lo, hi = np.array(scene.bounds["min"]), np.array(scene.bounds["max"])
    pts = (lo + (hi - lo) * rng.random((200, 3))).astype(np.float32)
    tris = lifted[i].astype(np.float32)
    fresh = quarry.Scene(tris)
    a, b = scene.closest(pts), fresh.closest(pts)
    assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])
    partial = tris.copy()
    dirty = np.array([0, 5, 7, 2047], np.int32)
    partial[dirty] += np.array([0.0, 3.0, 0.0], np.float32)
    scene.update_triangles(partial, dirty=dirty)
    assert scene.validate() == "" and scene.refit_stats["updated"] == 4
    fresh = quarry.Scene(partial)
    a, b = scene.closest(pts), fresh.closest(pts)
    assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])
    # topology: delete 3, append 150 -> bitwise equal to a fresh build
    deleted = np.array([3, 100, 700], np.int32)
    keep = np.ones(len(partial), bool)
    keep[deleted] = False
    extra = (lo + 0.2 * (hi - lo) * rng.random((150, 3, 3))).astype(np.float32)
    new_tris = np.concatenate([partial[keep], extra])
    topo = scene.update_topology(new_tris, deleted=deleted)
    assert topo["deleted"] == 3 and topo["appended"] == 150
    assert scene.triangle_count == len(new_tris) and scene.validate() == ""
    fresh = quarry.Scene(new_tris)
    for m in ("closest",):
        a, b = getattr(scene, m)(pts), getattr(fresh, m)(pts)
        assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])
    a, b = scene.knn(pts, 8), fresh.knn(pts, 8)
    assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])
    moved = new_tris.copy()
    ids = np.array([0, 5, 11], np.int32)
    moved[ids] += np.array([0.0, 0.5, 0.0], np.float32)
    mt = scene.update_topology(moved, moved=ids)
    assert not mt["full_rebuild"] and mt["refit_ms"] > 0 and scene.validate() == ""
    with pytest.raises(ValueError):
        scene.update_vertices(lifted)


def test_point_cloud_bitwise(cuda):
    rng = np.random.default_rng(11)
    pts = (rng.random((20000, 3)) * 50).astype(np.float32)
    cloud = quarry.PointCloud(pts)
    assert cloud.point_count == 20000 and cloud.validate() == ""
    q = (rng.random((200, 3)) * 50).astype(np.float32)
    diff = pts[None, :, :] - q[:, None, :]
    d2 = (diff * diff).sum(axis=-1, dtype=np.float32)
    best = d2.argmin(axis=1)
    cd2, cid = cloud.closest(q)
    assert np.array_equal(_bits(cd2), _bits(d2[np.arange(200), best]))
    assert np.array_equal(cid, best.astype(np.int32))
    kd, kid = cloud.knn(q, 4)
    for j in range(200):
        o = np.argsort(d2[j], kind="stable")[:4]
        assert np.array_equal(kid[j], o.astype(np.int32))
    r = 5.0
    off, rd2, rid = cloud.radius(q, r)
    for j in range(200):
        want = np.nonzero(d2[j] <= r * r)[0]
        want = want[np.argsort(d2[j][want], kind="stable")]
        assert np.array_equal(rid[off[j]:off[j + 1]], want.astype(np.int32))
    moved = pts.copy()
    moved[:, 1] += np.float32(0.1)
    cloud.update_points(moved)
    assert cloud.validate() == ""
    part = moved.copy()
    dirty = np.array([0, 3, 17, 19999], np.int32)
    part[dirty] += np.array([0.0, 0.5, 0.0], np.float32)
    cloud.update_points(part, dirty=dirty)
    assert cloud.validate() == "" and cloud.refit_stats["updated"] == 4
    pdel = np.array([0, 7, 10, 555], np.int32)
    keep = np.ones(20000, bool)
    keep[pdel] = False
    new_pts = np.concatenate([part[keep], (rng.random((500, 3)) * 50).astype(np.float32)])
    t = cloud.update_topology(new_pts, deleted=pdel)
    assert t["deleted"] == 4 and t["appended"] == 500 and cloud.validate() == ""
    fresh = quarry.PointCloud(new_pts)
    a, b = cloud.closest(q), fresh.closest(q)
    assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])
    sah = quarry.PointCloud(new_pts, builder="sah")
    a2 = sah.closest(q, order="morton", wide=True)
    assert np.array_equal(_bits(a2[0]), _bits(b[0])) and np.array_equal(a2[1], b[1])


def test_gaussian_cloud(cuda):
    m, r, s = quarry.demo_gaussians("sheet", 2000, seed=3)
    g = quarry.GaussianCloud(m, r, s)
    assert g.gaussian_count == 2000 and g.validate() == ""
    items = np.concatenate([m, r, s], axis=1).astype(np.float32)
    lo, hi = np.array(g.bounds["min"]), np.array(g.bounds["max"])
    q = (lo + (hi - lo) * np.random.default_rng(4).random((200, 3))).astype(np.float32)
    want = oracle.closest_brute("gauss", items, q)
    d2, idx = g.closest(q)
    assert np.array_equal(_bits(d2), want[:, 0]) and np.array_equal(idx, want[:, 1].view(np.int32))
    wk = oracle.knn_brute("gauss", items, q, 4)
    kd, kid = g.knn(q, 4, order="morton", wide=True)
    assert np.array_equal(_bits(kd), wk[..., 0]) and np.array_equal(kid, wk[..., 1].view(np.int32))
    g.update(m + np.float32(0.1), r, s)
    assert g.validate() == ""
    g.update(m + np.float32(0.1), r, s, dirty=np.array([0, 7], np.int32))
    assert g.validate() == "" and g.refit_stats["updated"] == 2


def test_bad_inputs_raise_value_error(mesh):
    v, i = mesh
    scene = quarry.Scene(v, i)
    face = quarry.Scene(v[i].astype(np.float32))
    pts = np.zeros((4, 3), np.float32)
    m, r, s = quarry.demo_gaussians("sheet", 50, seed=1)
    cloud = quarry.PointCloud(np.random.default_rng(1).random((100, 3)).astype(np.float32))
    bad = [
        lambda: quarry.Scene(np.zeros((5, 3), np.float32)),
        lambda: quarry.PointCloud(np.zeros((1, 3), np.float32)),
        lambda: scene.knn(pts, 0),
        lambda: scene.knn(pts, 33),
        lambda: cloud.knn(pts, 33),
        lambda: scene.raycast(pts, pts[:-1]),
        lambda: scene.update_triangles(v[i][:10].astype(np.float32)),
        lambda: cloud.update_points(np.zeros((10, 3), np.float32)),
        lambda: quarry.GaussianCloud(m, r, s[:10]),
        lambda: quarry.GaussianCloud(m, r, -s),
        lambda: face.update_vertices(v),
        lambda: scene.closest(pts, order="bogus"),
        lambda: quarry.Scene(v, i, builder="octree"),
        lambda: scene.radius(pts, -1.0),
        lambda: scene.update_topology(v[i].astype(np.float32), deleted=np.array([5, 3], np.int32)),
        lambda: scene.update_topology(v[i].astype(np.float32)[:-1]),
    ]
    for call in bad:
        with pytest.raises(ValueError):
            call()


def test_leaf_size_4_builder_through_the_module(mesh):
    """builder="sah4" (engine addition): the leaf-size-4 SAH tree, whose 4-wide layer is the
    leaf-range form, answers every query of every kind with the LBVH's bits, also after a
    refit and a topology edit."""
    v, i = mesh
    base, s4 = quarry.Scene(v, i), quarry.Scene(v, i, builder="sah4")
    assert s4.validate() == "" and s4.node_count == base.node_count
    assert "sah_bin_ms" in s4.build_stats
    lo, hi = np.array(base.bounds["min"]), np.array(base.bounds["max"])
    rng = np.random.default_rng(21)
    pts = (lo + (hi - lo) * rng.random((400, 3))).astype(np.float32)
    radius = 0.2 * float(np.max(hi - lo))

    def same(a, b, kw):
        for fn in (lambda s: s.closest(pts, **kw), lambda s: s.knn(pts, 4, **kw),
                   lambda s: s.radius(pts, radius, **kw)):
            x, y = fn(a), fn(b)
            for u, w in zip(x, y):
                assert np.array_equal(np.ascontiguousarray(u).view(np.uint8),
                                      np.ascontiguousarray(w).view(np.uint8)), kw

    for kw in ({}, {"wide": True}, {"order": "coherent", "wide": True}):
        same(s4, base, kw)
    origins = (lo + (hi - lo) * rng.random((300, 3))).astype(np.float32)
    origins[:, 1] = hi[1] + 1.0
    dirs = rng.normal(size=(300, 3)).astype(np.float32)
    dirs[:, 1] = -np.abs(dirs[:, 1]) - 0.5
    for kw in ({}, {"wide": True}):
        h1, t1 = s4.raycast(origins, dirs, **kw)
        h0, t0 = base.raycast(origins, dirs)
        assert np.array_equal(h1, h0) and np.array_equal(_bits(t1), _bits(t0))
    lifted = v.copy()
    lifted[:, 1] += np.float32(0.25)
    s4.update_vertices(lifted)
    base.update_vertices(lifted)
    assert s4.validate() == ""
    same(s4, base, {"wide": True})
    pr = np.random.default_rng(5)
    pc = (pr.random((5000, 3)) * 20).astype(np.float32)
    c4, c0 = quarry.PointCloud(pc, builder="sah4"), quarry.PointCloud(pc)
    q = (pr.random((300, 3)) * 20).astype(np.float32)
    for kw in ({}, {"wide": True}):
        a, b = c4.knn(q, 8, **kw), c0.knn(q, 8)
        assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])
    keep = np.ones(5000, bool)
    keep[[3, 99, 4000]] = False
    newp = np.concatenate([pc[keep], (pr.random((40, 3)) * 20).astype(np.float32)])
    c4.update_topology(newp, deleted=np.array([3, 99, 4000], np.int32))
    assert c4.validate() == ""
    fresh = quarry.PointCloud(newp)
    a, b = c4.closest(q, wide=True), fresh.closest(q)
    assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])
    m, r, s = quarry.demo_gaussians("sheet", 1500, seed=8)
    g4, g0 = quarry.GaussianCloud(m, r, s, builder="sah4"), quarry.GaussianCloud(m, r, s)
    gq = q * np.float32(0.1)
    a, b = g4.closest(gq, wide=True), g0.closest(gq)
    assert np.array_equal(_bits(a[0]), _bits(b[0])) and np.array_equal(a[1], b[1])
