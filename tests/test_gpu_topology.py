"""Topology edits (qk_update_topology, updateBVHGPU): subtree surgery gives a valid tree whose
query results are bit-identical to the oracle's and to a fresh build of the edited scene.

Edit scripts follow quarry's GpuTopoEdit (src/gpu/gpu_bvh.h:182-213): the new scene is the old
one's survivors in order, new primitives at `inserted` new indices, `appended` more at the end,
and `moved` new indices with changed geometry.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from quarry import capi, workloads

pytestmark = pytest.mark.gpu


def _dev(a, dtype=np.float32):
    return capi.to_device(np.ascontiguousarray(a), dtype)


def _items(kind, n, seed):
    if kind == "tri":
        return workloads.city(max(n // 10, 2), seed)[0]
    if kind == "point":
        return workloads.point_cloud("surface", n, seed)
    return workloads.gaussians(n, 0.05, 1.0, seed)


def _fresh(kind, items, rng, count):
    """New primitives near existing ones (copies of random primitives, shifted a little)."""
    src = items[rng.integers(0, len(items), count)].copy()
    shift = rng.normal(0, 0.5, (count, 3)).astype(np.float32)
    if kind == "tri":
        src += np.tile(shift, 3)
    else:
        src[:, :3] += shift
    return src


def _move(kind, rows, rng):
    rows = rows.copy()
    shift = rng.normal(0, 0.05, (len(rows), 3)).astype(np.float32)
    if kind == "tri":
        rows += np.tile(shift, 3)
    else:
        rows[:, :3] += shift
    return rows


def make_edit(kind, items, rng, n_del, n_ins, n_app, n_mov, deleted=None):
    """(new scene, deleted, inserted, moved) of a random edit script."""
    n_old = len(items)
    if deleted is None:
        deleted = np.sort(rng.choice(n_old, n_del, replace=False)).astype(np.int32)
    survivors = np.delete(items, deleted, axis=0)
    n_new = n_old - len(deleted) + n_ins + n_app
    tail = n_new - n_app
    inserted = np.sort(rng.choice(tail, n_ins, replace=False)).astype(np.int32)
    new = np.empty((n_new, items.shape[1]), np.float32)
    keep = np.ones(tail, bool)
    keep[inserted] = False
    new[:tail][keep] = survivors
    new[inserted] = _fresh(kind, items, rng, n_ins)
    new[tail:] = _fresh(kind, items, rng, n_app)
    moved = np.sort(rng.choice(n_new, n_mov, replace=False)).astype(np.int32)
    new[moved] = _move(kind, new[moved], rng)
    return new, deleted, inserted, moved


def _queries(items, kind, n, seed):
    if kind == "tri":
        lo, hi = workloads.bounds_of(items)
    else:
        lo, hi = items[:, :3].min(0), items[:, :3].max(0)
    return workloads.uniform_points(n, lo - 1.0, hi + 1.0, seed, 21)


def _same_results(tree, kind, items, seed, fresh=None):
    """Closest / kNN / radius (and rays for triangles) equal the oracle's on `items`."""
    ref = oracle.LBVH(kind, items)
    q = _queries(items, kind, 1_500, seed)
    dq = _dev(q)
    assert np.array_equal(tree.closest(dq).cpu().numpy().view(np.uint32), ref.closest(q))
    assert np.array_equal(tree.knn(dq, 8).cpu().numpy().view(np.uint32), ref.knn(q, 8))
    lo, hi = q.min(0), q.max(0)
    r = float(np.linalg.norm(hi - lo)) * 0.03
    off, keys = tree.radius(dq, r)
    woff, wkeys = ref.radius(q, r)
    assert np.array_equal(off.cpu().numpy().astype(np.int64), woff)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), wkeys)
    if kind == "tri":
        blo, bhi = workloads.bounds_of(items)
        rays = workloads.cosine_rays(20_000, float(blo[0]), float(bhi[0]), float(blo[1]),
                                     float(bhi[1]), float(bhi[2]) + 5.0, seed)
        got = tree.raycast(_dev(rays)).cpu().numpy().view(np.uint64)
        assert np.array_equal(got, ref.raycast(rays))
        if fresh is not None:
            assert np.array_equal(got, fresh.raycast(_dev(rays)).cpu().numpy().view(np.uint64))


CASES = [("tri", 30_000), ("point", 40_000), ("gauss", 12_000)]


@pytest.mark.parametrize("kind,n", CASES)
@pytest.mark.parametrize("builder", ["lbvh", "sah"])
def test_surgery_matches_oracle(cuda, kind, n, builder):
    rng = np.random.default_rng(7)
    items = _items(kind, n, 3)
    tree = capi.DeviceTree(kind, items, builder=builder)
    new, dele, ins, mov = make_edit(kind, items, rng, 60, 25, 40, 30)
    info = tree.update_topology(new, dele, ins, mov)
    assert info["rebuild"] == 0, info
    assert info["cuts"] > 0 and info["new_leaves"] < len(new) // 4
    assert tree.n == len(new)
    assert tree.validate() == [0] * 8
    _same_results(tree, kind, new, 11, capi.DeviceTree(kind, new, builder=builder))


@pytest.mark.parametrize("kind,n", CASES)
def test_surgery_repeated_edits(cuda, kind, n):
    """Edits on trees that earlier edits reshaped (slots no longer in build order)."""
    rng = np.random.default_rng(17)
    items = _items(kind, n, 5)
    tree = capi.DeviceTree(kind, items, builder="sah")
    for step in range(4):
        new, dele, ins, mov = make_edit(kind, items, rng, 40 + 10 * step, 20, 15 * step, 10)
        info = tree.update_topology(new, dele, ins, mov)
        assert info["rebuild"] == 0, (step, info)
        assert tree.validate() == [0] * 8
        items = new
    _same_results(tree, kind, items, 13)


@pytest.mark.parametrize("shape", ["delete_only", "append_only", "insert_only", "one_each"])
def test_surgery_edit_shapes(cuda, shape):
    rng = np.random.default_rng(23)
    items = _items("point", 20_000, 9)
    tree = capi.DeviceTree("point", items)
    counts = {"delete_only": (100, 0, 0, 0), "append_only": (0, 0, 300, 0),
              "insert_only": (0, 200, 0, 0), "one_each": (1, 1, 1, 1)}[shape]
    new, dele, ins, mov = make_edit("point", items, rng, *counts)
    info = tree.update_topology(new, dele, ins, mov)
    assert info["rebuild"] == 0, info
    assert tree.validate() == [0] * 8
    _same_results(tree, "point", new, 3)


@pytest.mark.parametrize("cut", [2, 16, 64, 0])
def test_surgery_contiguous_delete_splices(cuda, cut):
    """Deleting whole subtrees empties cuts: their parents are spliced out."""
    rng = np.random.default_rng(29)
    items = _items("point", 30_000, 4)
    tree = capi.DeviceTree("point", items)
    # scene indices of a run of consecutive leaf slots: whole subtrees
    prim = tree.host("prim_ids", np.int32, tree.n)
    dele = np.sort(prim[5_000:5_700]).astype(np.int32)
    new, dele, ins, mov = make_edit("point", items, rng, 0, 10, 10, 5, deleted=dele)
    info = tree.update_topology(new, dele, ins, mov, cut_size=cut)
    assert info["rebuild"] == 0 and info["spliced"] > 0, info
    assert tree.validate() == [0] * 8
    _same_results(tree, "point", new, 5)


@pytest.mark.parametrize("kind", ["tri", "point"])
def test_surgery_cut_grows_past_a_warp(cuda, kind):
    """New primitives all landing in one cut push it past 256 primitives (the warp builder's
    largest range): the block builder takes that subtree.  quarry's examples/dynamic_scene.cpp
    makes such edits (props appended next to a cut of about 256 leaves)."""
    rng = np.random.default_rng(41)
    items = _items(kind, 40_000, 12)
    tree = capi.DeviceTree(kind, items, builder="lbvh")
    extra = np.repeat(items[100:101], 200, axis=0)
    shift = rng.normal(0, 1e-3, (200, 3)).astype(np.float32)
    if kind == "tri":
        extra += np.tile(shift, 3)
    else:
        extra[:, :3] += shift
    new = np.concatenate([items, extra]).astype(np.float32)
    info = tree.update_topology(new, [], [], [], cut_size=250)
    assert info["rebuild"] == 0, info
    assert info["max_cut"] > 256, info
    assert tree.validate() == [0] * 8
    _same_results(tree, kind, new, 17, capi.DeviceTree(kind, new))


def test_surgery_declines_large_edits(cuda):
    rng = np.random.default_rng(31)
    items = _items("point", 8_000, 6)
    tree = capi.DeviceTree("point", items)
    new, dele, ins, mov = make_edit("point", items, rng, 3_000, 0, 0, 0)
    info = tree.update_topology(new, dele, ins, mov)
    assert info["rebuild"] == 1 and info["reason"] in (1, 2, 4), info
    assert tree.validate() == [0] * 8
    _same_results(tree, "point", new, 7)
    # a tree that is a single cut (root of at most cut_size leaves)
    small = capi.DeviceTree("point", items[:100])
    new2, d2, i2, m2 = make_edit("point", items[:100], rng, 3, 0, 0, 0)
    info = small.update_topology(new2, d2, i2, m2, cut_size=256)
    assert info["rebuild"] == 1 and info["reason"] == 1


def test_surgery_deterministic(cuda):
    rng = np.random.default_rng(37)
    items = _items("tri", 20_000, 8)
    new, dele, ins, mov = make_edit("tri", items, rng, 50, 30, 30, 20)
    a = capi.DeviceTree("tri", items, builder="sah")
    b = capi.DeviceTree("tri", items, builder="sah")
    a.update_topology(new, dele, ins, mov)
    b.update_topology(new, dele, ins, mov)
    assert a.nodes_bytes().tobytes() == b.nodes_bytes().tobytes()
    assert np.array_equal(a.host("prim_ids", np.int32, a.n), b.host("prim_ids", np.int32, b.n))


def test_surgery_invalid_scripts(cuda):
    items = _items("point", 5_000, 2)
    tree = capi.DeviceTree("point", items)
    with pytest.raises(capi.QkError):
        tree.update_topology(items[:-1], deleted=[3, 2], inserted=[0])  # not ascending
    tree = capi.DeviceTree("point", items)
    with pytest.raises(capi.QkError):
        tree.update_topology(items[:-1], deleted=[len(items)])  # out of range


def test_python_update_topology_uses_surgery(cuda):
    """The module's update_topology (C++ updateBVHGPU) takes the surgery path on small edits
    and answers like a freshly built Scene."""
    import quarry

    rng = np.random.default_rng(41)
    tris = _items("tri", 30_000, 12)
    scene = quarry.Scene(tris.reshape(-1, 3, 3), builder="sah")
    new, dele, ins, mov = make_edit("tri", tris, rng, 40, 20, 20, 10)
    tm = scene.update_topology(new.reshape(-1, 3, 3), deleted=dele, moved=mov, inserted=ins)
    assert tm["full_rebuild"] is False and tm["surgery_roots"] > 0, tm
    assert scene.triangle_count == len(new)
    assert scene.validate() == ""
    fresh = quarry.Scene(new.reshape(-1, 3, 3), builder="sah")
    q = _queries(new, "tri", 2_000, 3)
    for a, b in zip(scene.closest(q), fresh.closest(q)):
        assert np.array_equal(a, b)
    lo, hi = workloads.bounds_of(new)
    rays = workloads.cosine_rays(10_000, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                                 float(hi[2]) + 5.0, 4)
    for a, b in zip(scene.raycast(rays[:, :3], rays[:, 3:6]),
                    fresh.raycast(rays[:, :3], rays[:, 3:6])):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("kind", ["point", "gauss"])
def test_python_clouds_update_topology_rounds(cuda, kind):
    """PointCloud / GaussianCloud.update_topology (updatePointBVHGPU / updateGaussianBVHGPU):
    three mixed edits in a row on one object (the C++ layer reuses its spare arrays and keeps
    the 4-wide layer), each answering like a freshly built object, wide queries included."""
    import quarry

    rng = np.random.default_rng(43)
    items = _items(kind, 20_000, 14)

    def make(a):
        if kind == "point":
            return quarry.PointCloud(a)
        return quarry.GaussianCloud(a[:, :3].copy(), a[:, 3:7].copy(), a[:, 7:10].copy())

    def update(obj, a, dele, ins, mov):
        if kind == "point":
            return obj.update_topology(a, deleted=dele, moved=mov, inserted=ins)
        return obj.update_topology(a[:, :3].copy(), a[:, 3:7].copy(), a[:, 7:10].copy(),
                                   deleted=dele, moved=mov, inserted=ins)

    obj = make(items)
    lo, hi = items[:, :3].min(0), items[:, :3].max(0)
    q = workloads.uniform_points(1_000, lo - 1.0, hi + 1.0, 5, 21)
    obj.closest(q, wide=True)  # builds the 4-wide layer
    for step in range(3):
        new, dele, ins, mov = make_edit(kind, items, rng, 30, 15, 10 + 5 * step, 20)
        tm = update(obj, new, dele, ins, mov)
        assert tm["full_rebuild"] is False, (step, tm)
        assert obj.validate() == ""
        fresh = make(new)
        for wide in (False, True):
            for a, b in zip(obj.closest(q, wide=wide), fresh.closest(q, wide=wide)):
                assert np.array_equal(a, b), (step, wide)
            for a, b in zip(obj.knn(q, 8, wide=wide), fresh.knn(q, 8, wide=wide)):
                assert np.array_equal(a, b), (step, wide)
        for a, b in zip(obj.radius(q, 2.0), fresh.radius(q, 2.0)):
            assert np.array_equal(a, b), step
        items = new
