"""GPU parity of the engine through its C ABI (quarry.capi) against the oracle.

Every check is bit-exact: node arrays and tree hashes against the oracle's restatement of
the reference LBVH, ray results as (hit << 32 | bits(t)), query results as (dist2 bits, id),
radius CSR keys, for binary and 4-wide traversal, input and Morton order.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from quarry import capi, workloads

pytestmark = pytest.mark.gpu

FLAG_SETS = [0, capi.QK_ORDER_MORTON, capi.QK_WIDE, capi.QK_ORDER_MORTON | capi.QK_WIDE,
             capi.QK_ORDER_COHERENT, capi.QK_ORDER_COHERENT | capi.QK_WIDE]


def _dev(a, dtype=np.float32):
    return capi.to_device(np.ascontiguousarray(a), dtype)


def _random_rays(lo, hi, n, seed):
    """Rays from a sphere around the box toward jittered targets (some miss)."""
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


def _scenes():
    terrain = workloads.terrain(48, 3)
    mixed = workloads.demo_mesh_tris(2, 24, 1500, 7, 0)
    city, _ = workloads.city(300, 5)
    return {"terrain": terrain, "mixed": mixed, "city": city}


SCENES = None


def scenes():
    global SCENES
    if SCENES is None:
        SCENES = _scenes()
    return SCENES


def _check_tree(tree: capi.DeviceTree, ref: oracle.LBVH):
    n = tree.n
    got_nodes = tree.nodes_bytes()
    assert got_nodes.tobytes() == ref.nodes.tobytes(), "node array differs from the oracle"
    assert np.array_equal(tree.host("prim_ids", np.int32, n), ref.prim_ids)
    assert np.array_equal(tree.host("depth_arr", np.int32, 2 * n - 1), ref.depth_arr)
    assert tree.depth == ref.depth
    assert tree.validate() == [0] * 8


# ---------------------------------------------------------------------------------------
# radix sort
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("n,bits", [(1, 8), (5, 30), (4096, 30), (4097, 30), (100_000, 32),
                                    (300_000, 30)])
def test_sort_pairs_stable(cuda, n, bits):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 2 ** bits if bits < 32 else 2 ** 32, size=n, dtype=np.uint64)
    keys[: n // 3] = keys[0]  # many duplicates exercise stability
    keys = keys.astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    kd, vd = capi.sort_pairs(_dev(keys.view(np.int32), np.int32), _dev(vals.view(np.int32), np.int32), bits)
    order = np.argsort(keys & np.uint32((1 << bits) - 1 if bits < 32 else 0xFFFFFFFF), kind="stable")
    assert np.array_equal(vd.cpu().numpy().view(np.uint32), vals[order])
    assert np.array_equal(kd.cpu().numpy().view(np.uint32), keys[order])


# ---------------------------------------------------------------------------------------
# LBVH build == the reference algorithm (oracle restatement), bit for bit
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["terrain", "mixed", "city"])
def test_lbvh_triangles_match_oracle(cuda, name):
    tris = scenes()[name]
    tree = capi.DeviceTree("tri", tris)
    _check_tree(tree, oracle.LBVH("tri", tris))


@pytest.mark.parametrize("kind,n", [("point", 2), ("point", 3), ("point", 1000),
                                    ("point", 50_000), ("gauss", 2), ("gauss", 5000)])
def test_lbvh_points_gaussians_match_oracle(cuda, kind, n):
    if kind == "point":
        items = workloads.point_cloud("volume", n, 11)
    else:
        items = workloads.gaussians(n, 0.05, 1.0, 11)
    tree = capi.DeviceTree(kind, items)
    _check_tree(tree, oracle.LBVH(kind, items))


def test_lbvh_duplicate_positions(cuda):
    """All-coincident and repeated points: equal Morton codes ordered by index."""
    pts = np.zeros((777, 3), np.float32)
    pts[::3] = [1.0, 2.0, 3.0]
    tree = capi.DeviceTree("point", pts)
    _check_tree(tree, oracle.LBVH("point", pts))


def test_wide_nodes_match_oracle(cuda):
    tris = scenes()["terrain"]
    tree = capi.DeviceTree("tri", tris)
    count = tree.build_wide()
    ref = oracle.LBVH("tri", tris)
    wide, wide_id = ref.wide()
    assert count == len(wide) // 4
    got = tree.arrays["wide"].cpu().numpy()[: count * 128]
    assert got.tobytes() == wide.tobytes()
    assert np.array_equal(tree.host("wide_id", np.int32, tree.n - 1), wide_id)
    assert tree.validate() == [0] * 8


# ---------------------------------------------------------------------------------------
# rays
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["terrain", "mixed", "city"])
def test_raycast_parity(cuda, name):
    tris = scenes()[name]
    lo, hi = workloads.bounds_of(tris)
    ref = oracle.LBVH("tri", tris)
    tree = capi.DeviceTree("tri", tris)
    tree.build_wide()
    ray_sets = [
        workloads.down_rays(20_000, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                            float(hi[2]) + 10.0, 9),
        _random_rays(lo, hi, 20_000, 10),
        workloads.cosine_rays(20_000, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                              float(hi[2]) + 5.0, 12),
    ]
    for rays in ray_sets:
        want = ref.raycast(rays)
        d_rays = _dev(rays)
        for flags in FLAG_SETS + [capi.QK_ORDER_DIRECTION, capi.QK_ORDER_DIRECTION | capi.QK_WIDE]:
            got = tree.raycast(d_rays, flags).cpu().numpy().view(np.uint64)
            assert np.array_equal(got, want), f"flags={flags}: {(got != want).sum()} rays differ"


def test_degenerate_rays_every_ray_path(cuda):
    """Rays with tmin / tmax not NaN and no parallel axis, or only x and y parallel
    (vertical), take traversals compiled for that case (no branch on parallel axes, min / max
    slab updates); the others (one parallel axis of x / y, |d| < 1e-20 components, zero
    directions, NaN tmin or tmax) keep the general one.  A mix of all, with infinite tmax,
    negative tmin and origins inside the scene, through every binary and 4-wide ray schedule
    and order, gives the oracle's bits."""
    tris = scenes()["city"]
    lo, hi = workloads.bounds_of(tris)
    rays = _random_rays(lo, hi, 20_000, 31)
    rng = np.random.default_rng(8)
    rays[0::7, 3] = 0.0                   # parallel to x
    rays[1::7, 4] = 0.0                   # parallel to y
    rays[2::7, 3:5] = 0.0                 # vertical
    rays[3::7, 5] = 1e-21                 # a tiny component counts as parallel
    rays[4::7, 3:6] = 0.0                 # no direction at all
    rays[5::11, 6] = np.nan               # NaN tmin
    rays[6::11, 7] = np.nan               # NaN tmax
    rays[7::11, 7] = np.inf               # unbounded
    rays[8::11, 6] = -5.0                 # negative tmin
    inside = np.arange(9, len(rays), 13)
    rays[inside, :3] = (lo + (hi - lo) * rng.random((len(inside), 3))).astype(np.float32)
    want = oracle.LBVH("tri", tris).raycast(rays)
    assert np.count_nonzero(want >> 32) > 1_000
    d_rays = _dev(rays)
    for builder in ("lbvh", "sah"):
        tree = capi.DeviceTree("tri", tris, builder=builder)
        tree.build_wide()
        occ, coh = capi.QK_TUNE_HIGH_OCC, capi.QK_ORDER_COHERENT
        for flags in (0, occ, coh | occ, capi.QK_ORDER_MORTON, capi.QK_TUNE_DYNAMIC,
                      capi.QK_TUNE_SHORT_STACK, occ | capi.QK_TUNE_LEAF4, capi.QK_WIDE,
                      capi.QK_WIDE | coh):
            got = tree.raycast(d_rays, flags).cpu().numpy().view(np.uint64)
            assert np.array_equal(got, want), (builder, flags, int((got != want).sum()))


def test_ordered_raycast_captures_in_a_cuda_graph(cuda):
    """The ordering passes and the traversal after them launch with programmatic stream
    serialization; captured into a CUDA graph and replayed they give the same bits."""
    tris = scenes()["city"]
    lo, hi = workloads.bounds_of(tris)
    rays = _dev(workloads.cosine_rays(70_001, float(lo[0]), float(hi[0]), float(lo[1]),
                                      float(hi[1]), float(hi[2]) + 5.0, 3))
    tree = capi.DeviceTree("tri", tris, builder="sah")
    for flags in (capi.QK_ORDER_COHERENT | capi.QK_TUNE_HIGH_OCC, capi.QK_ORDER_COHERENT,
                  capi.QK_ORDER_MORTON | capi.QK_TUNE_HIGH_OCC):
        want = tree.raycast(rays, 0).clone()
        out = cuda.empty_like(want)
        ws = cuda.empty(capi.lib().qk_query_workspace_bytes(rays.shape[0], flags),
                        dtype=cuda.uint8, device="cuda")
        side = cuda.cuda.Stream()
        side.wait_stream(cuda.cuda.current_stream())
        with cuda.cuda.stream(side):
            tree.raycast(rays, flags, out=out, ws=ws)  # warm-up outside the capture
        cuda.cuda.current_stream().wait_stream(side)
        g = cuda.cuda.CUDAGraph()
        out.zero_()
        with cuda.cuda.graph(g):
            tree.raycast(rays, flags, out=out, ws=ws)
        for _ in range(3):
            out.zero_()
            g.replay()
            cuda.cuda.synchronize()
            assert cuda.equal(out, want), flags


def test_raycast_stats_and_no_overflow(cuda):
    tris = scenes()["terrain"]
    tree = capi.DeviceTree("tri", tris)
    lo, hi = workloads.bounds_of(tris)
    rays = workloads.down_rays(5000, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]), 50.0, 3)
    stats = cuda.zeros(4, dtype=cuda.int64, device="cuda")
    tree.raycast(_dev(rays), 0, stats=stats)
    s = stats.cpu().numpy()
    assert s[0] > 5000 and s[1] >= 5000 and s[2] == 0


# ---------------------------------------------------------------------------------------
# point queries over the three primitive kinds
# ---------------------------------------------------------------------------------------
def _items(kind):
    if kind == "tri":
        return scenes()["mixed"]
    if kind == "point":
        return workloads.point_cloud("sphere", 30_000, 4)
    return workloads.gaussians(6000, 0.05, 1.0, 4)


def _queries(items, kind, n, seed):
    if kind == "tri":
        lo, hi = workloads.bounds_of(items)
    else:
        lo, hi = items[:, :3].min(0), items[:, :3].max(0)
    return workloads.uniform_points(n, lo - 1.0, hi + 1.0, seed, 21)


@pytest.mark.parametrize("kind", ["tri", "point", "gauss"])
def test_closest_knn_parity(cuda, kind):
    items = _items(kind)
    q = _queries(items, kind, 4000, 5)
    ref = oracle.LBVH(kind, items)
    tree = capi.DeviceTree(kind, items)
    tree.build_wide()
    dq = _dev(q)
    want_c = ref.closest(q)
    for flags in FLAG_SETS:
        got = tree.closest(dq, flags).cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want_c), f"closest flags={flags}"
    for k in (1, 3, 8, 16, 32):
        want_k = ref.knn(q, k)
        for flags in FLAG_SETS:
            got = tree.knn(dq, k, flags).cpu().numpy().view(np.uint32)
            assert np.array_equal(got, want_k), f"knn k={k} flags={flags}"
    # wider stride than k pads only the first k entries of each row
    got = tree.knn(dq, 5, 0, stride=9).cpu().numpy().view(np.uint32)
    assert np.array_equal(got[:, :5], ref.knn(q, 5))


@pytest.mark.parametrize("kind,r", [("tri", 2.5), ("point", 4.0), ("gauss", 1.5),
                                    ("point", 0.0), ("point", 40.0)])
def test_radius_parity(cuda, kind, r):
    items = _items(kind)
    q = _queries(items, kind, 1500, 6)
    ref = oracle.LBVH(kind, items)
    want_off, want_keys = ref.radius(q, r)
    tree = capi.DeviceTree(kind, items)
    tree.build_wide()
    dq = _dev(q)
    for flags in FLAG_SETS:
        off, keys = tree.radius(dq, r, flags)
        off = off.cpu().numpy().astype(np.int64)
        keys = keys.cpu().numpy().view(np.uint64)
        assert np.array_equal(off, want_off), f"offsets flags={flags}"
        assert np.array_equal(keys, want_keys), f"keys flags={flags}"


# ---------------------------------------------------------------------------------------
# refit
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("kind", ["tri", "point", "gauss"])
def test_refit_full_and_dirty(cuda, kind):
    items = _items(kind).copy()
    tree = capi.DeviceTree(kind, items)
    tree.build_wide()
    ref = oracle.LBVH(kind, items)
    rng = np.random.default_rng(3)
    moved = items.copy()
    moved[:, :3] += rng.normal(0, 0.05, size=(len(items), 3)).astype(np.float32)
    if kind == "tri":
        moved[:, 3:9] += rng.normal(0, 0.05, size=(len(items), 6)).astype(np.float32)
    tree.refit(moved)
    ref.refit(moved)
    assert tree.nodes_bytes().tobytes() == ref.nodes.tobytes()
    assert tree.validate() == [0] * 8
    # partial: move a subset (with a repeated id) and refit only those
    ids = np.unique(rng.integers(0, len(items), size=max(3, len(items) // 100))).astype(np.int32)
    again = moved.copy()
    again[ids, :3] += np.float32(0.5)
    dup = np.concatenate([ids, ids[:1]])
    tree.refit_dirty(dup, again[dup])
    tree.items_scene = _dev(again)
    ref.refit(again)
    assert tree.nodes_bytes().tobytes() == ref.nodes.tobytes()
    assert tree.validate() == [0] * 8
    q = _queries(again, kind, 1000, 8)
    for flags in (0, capi.QK_WIDE):
        got = tree.closest(_dev(q), flags).cpu().numpy().view(np.uint32)
        assert np.array_equal(got, ref.closest(q))


# ---------------------------------------------------------------------------------------
# binned SAH builder: a different tree, identical query results
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("kind,n,bins", [("tri", None, 16), ("tri", None, 32), ("point", 2, 32),
                                         ("point", 3, 8), ("point", 700, 32),
                                         ("point", 60_000, 32), ("gauss", 5000, 64)])
def test_sah_tree_valid_and_results_identical(cuda, kind, n, bins):
    if kind == "tri":
        items = scenes()["city"]
    elif kind == "point":
        items = workloads.point_cloud("sphere", n, 5)
    else:
        items = workloads.gaussians(n, 0.05, 1.0, 5)
    tree = capi.DeviceTree(kind, items, builder="sah", sah_bins=bins)
    assert tree.validate() == [0] * 8
    assert tree.depth <= 62
    again = capi.DeviceTree(kind, items, builder="sah", sah_bins=bins)
    assert again.nodes_bytes().tobytes() == tree.nodes_bytes().tobytes(), "SAH not deterministic"
    ref = oracle.LBVH(kind, items)
    if kind == "tri":
        lo, hi = workloads.bounds_of(items)
    else:
        lo, hi = items[:, :3].min(0), items[:, :3].max(0)
    q = workloads.uniform_points(2000, lo - 1, hi + 1, 3, 21)
    tree.build_wide()
    assert tree.validate() == [0] * 8
    dq = _dev(q)
    for flags in FLAG_SETS:
        assert np.array_equal(tree.closest(dq, flags).cpu().numpy().view(np.uint32), ref.closest(q))
        assert np.array_equal(tree.knn(dq, 8, flags).cpu().numpy().view(np.uint32), ref.knn(q, 8))
    r = 3.0 if kind != "gauss" else 1.0
    off, keys = tree.radius(dq, r)
    woff, wkeys = ref.radius(q, r)
    assert np.array_equal(off.cpu().numpy().astype(np.int64), woff)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), wkeys)
    if kind == "tri":
        rays = workloads.cosine_rays(20_000, float(lo[0]), float(hi[0]), float(lo[1]),
                                     float(hi[1]), float(hi[2]) + 5.0, 8)
        want = ref.raycast(rays)
        for flags in FLAG_SETS:
            got = tree.raycast(_dev(rays), flags).cpu().numpy().view(np.uint64)
            assert np.array_equal(got, want)


def test_sah_city_large(cuda):
    """The benchmark city at reduced size exercises the global SAH tier (> 1024 primitives
    per range over several levels)."""
    tris, top = workloads.city(20_000, 1)
    tree = capi.DeviceTree("tri", tris, builder="sah", sah_bins=32)
    assert tree.validate() == [0] * 8
    lo, hi = workloads.bounds_of(tris)
    rays = workloads.cosine_rays(50_000, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                                 top + 50.0, 2)
    ref = oracle.LBVH("tri", tris)
    got = tree.raycast(_dev(rays)).cpu().numpy().view(np.uint64)
    assert np.array_equal(got, ref.raycast(rays))
    # the refit path works on SAH trees too
    moved = tris.copy()
    moved[:, 2::3] += np.float32(0.25)
    tree.refit(moved)
    ref.refit(moved)
    assert tree.validate() == [0] * 8
    got = tree.raycast(_dev(rays)).cpu().numpy().view(np.uint64)
    assert np.array_equal(got, ref.raycast(rays))


def test_raycast_host_pipeline_matches(cuda):
    tris = scenes()["city"]
    lo, hi = workloads.bounds_of(tris)
    tree = capi.DeviceTree("tri", tris, builder="sah")
    rays = workloads.cosine_rays(70_001, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                                 float(hi[2]) + 5.0, 3)
    want = tree.raycast(_dev(rays), capi.QK_ORDER_MORTON).cpu().numpy().view(np.uint64)
    host_rays = cuda.from_numpy(rays).pin_memory()
    one = cuda.cuda.Stream()
    for chunks, streams in ((1, None), (3, None), (8, None), (32, None), (5, (one,) * 4)):
        host_out = cuda.zeros(len(rays), dtype=cuda.int64).pin_memory()
        dev_rays = cuda.empty((len(rays), 8), dtype=cuda.float32, device="cuda")
        dev_out = cuda.empty(len(rays), dtype=cuda.int64, device="cuda")
        streams = tree.raycast_host(host_rays, host_out, dev_rays, dev_out,
                                    capi.QK_ORDER_MORTON, chunks, streams)
        # the read-back stream's last copy depends on every earlier step
        streams[3].synchronize()
        assert np.array_equal(host_out.numpy().view(np.uint64), want)
        cuda.cuda.synchronize()
        # without dev_out the traversals store into the pinned host_out themselves
        host_out.zero_()
        streams = tree.raycast_host(host_rays, host_out, dev_rays, None, 0, chunks, streams)
        streams[3].synchronize()
        assert np.array_equal(host_out.numpy().view(np.uint64), want)
        cuda.cuda.synchronize()
    with pytest.raises(RuntimeError):  # pageable host_out cannot take direct stores
        tree.raycast_host(host_rays, cuda.zeros(len(rays), dtype=cuda.int64), dev_rays, None, 0, 4)


def test_raycast_mapped_matches(cuda):
    """Zero-copy rays: the traversal reads pinned host rays and writes pinned host results;
    same bits as the device-resident call for input, Morton and coherent order; pageable
    memory is refused before any launch."""
    tris = scenes()["city"]
    lo, hi = workloads.bounds_of(tris)
    tree = capi.DeviceTree("tri", tris, builder="sah")
    rays = workloads.cosine_rays(40_001, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                                 float(hi[2]) + 5.0, 9)
    want = tree.raycast(_dev(rays), 0).cpu().numpy()
    host_rays = cuda.from_numpy(rays).pin_memory()
    for flags in (0, capi.QK_ORDER_MORTON, capi.QK_ORDER_COHERENT | capi.QK_TUNE_HIGH_OCC):
        host_out = cuda.zeros(len(rays), dtype=cuda.int64).pin_memory()
        tree.raycast_mapped(host_rays, host_out, flags)
        cuda.cuda.synchronize()
        assert np.array_equal(host_out.numpy(), want)
    pageable = cuda.zeros(len(rays), dtype=cuda.int64)
    with pytest.raises(RuntimeError):
        tree.raycast_mapped(cuda.from_numpy(rays), pageable, 0)
    with pytest.raises(RuntimeError):
        tree.raycast_mapped(host_rays, pageable, 0)


@pytest.mark.parametrize("tune", ["dyn", "occ", "dyn_occ", "sm", "occ_sm"])
@pytest.mark.parametrize("order", [0, capi.QK_ORDER_MORTON, capi.QK_ORDER_COHERENT])
def test_raycast_tuning_flags_same_bits(cuda, tune, order):
    tris = scenes()["city"]
    lo, hi = workloads.bounds_of(tris)
    tree = capi.DeviceTree("tri", tris, builder="sah")
    rays = workloads.cosine_rays(50_003, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                                 float(hi[2]) + 5.0, 11)
    flags = {"dyn": capi.QK_TUNE_DYNAMIC, "occ": capi.QK_TUNE_HIGH_OCC,
             "dyn_occ": capi.QK_TUNE_DYNAMIC | capi.QK_TUNE_HIGH_OCC,
             "sm": capi.QK_TUNE_SHORT_STACK,
             "occ_sm": capi.QK_TUNE_HIGH_OCC | capi.QK_TUNE_SHORT_STACK}[tune]
    flags |= order
    rd = _dev(rays)
    want, want_ids = tree.raycast_ids(rd, 0)
    got, got_ids = tree.raycast_ids(rd, flags)
    assert cuda.equal(got, want) and cuda.equal(got_ids, want_ids)
    stats = cuda.zeros(4, dtype=cuda.int64, device="cuda")
    tree.raycast(rd, flags, stats=stats)
    base = cuda.zeros(4, dtype=cuda.int64, device="cuda")
    tree.raycast(rd, 0, stats=base)
    # same traversal per ray: identical node and triangle test counts
    assert stats[:3].tolist() == base[:3].tolist()


@pytest.mark.parametrize("count", [0, 1, 63, 64, 65, 8191, 8192, 70_001])
def test_coherent_order_same_bits(cuda, count):
    """QK_ORDER_COHERENT (a counting sort on origin / direction or position keys) returns the
    input order's bits for rays, closest, kNN and radius: below 64 records (input order), at
    the bucket-count steps, with flat axes (a common origin; identical query points) and
    with non-finite coordinates in the batch."""
    tris = scenes()["city"]
    lo, hi = workloads.bounds_of(tris)
    tree = capi.DeviceTree("tri", tris, builder="sah")
    rays = workloads.cosine_rays(max(count, 1), float(lo[0]), float(hi[0]), float(lo[1]),
                                 float(hi[1]), float(hi[2]) + 5.0, 5)[:count]
    rng = np.random.default_rng(count)
    pts = rng.uniform(lo - 2, hi + 2, (count, 3)).astype(np.float32)
    if count >= 64:
        rays[: count // 3, :3] = rays[0, :3]   # a third share one origin
        pts[: count // 4] = pts[0]            # a quarter of the queries coincide
        rays[1, 0] = np.nan
        pts[2, 1] = np.inf
    variants = [(rays, pts)]
    if count >= 64:
        flat = rays.copy()
        flat[:, :3] = flat[0, :3]             # every origin equal: three flat axes
        same = np.repeat(pts[:1], count, axis=0)
        variants.append((flat, same))
    for r, p in variants:
        rd, pd = _dev(r), _dev(p)
        assert cuda.equal(tree.raycast(rd, capi.QK_ORDER_COHERENT), tree.raycast(rd, 0))
        assert cuda.equal(tree.raycast(rd, capi.QK_ORDER_COHERENT | capi.QK_TUNE_DYNAMIC),
                          tree.raycast(rd, 0))
        if count == 0:
            continue
        assert cuda.equal(tree.closest(pd, capi.QK_ORDER_COHERENT), tree.closest(pd, 0))
        assert cuda.equal(tree.knn(pd, 4, capi.QK_ORDER_COHERENT), tree.knn(pd, 4, 0))
        want = tree.radius(pd, 3.0, 0)
        got = tree.radius(pd, 3.0, capi.QK_ORDER_COHERENT | capi.QK_TUNE_STASH)
        assert all(cuda.equal(a, b) for a, b in zip(got, want))


@pytest.mark.parametrize("kind", ["tri", "point", "gauss"])
@pytest.mark.parametrize("n", [2, 3, 5, 40, 20_000])
def test_split_queries_same_bits(cuda, kind, n):
    """One warp per query over 32 disjoint subtrees, and groups of 8 and 4 lanes over 8 and 4
    subtrees: closest, kNN (k from 1 to 16: groups grow to k lanes) and radius equal the
    one-thread-per-query kernels, including trees shallower than the split levels and a query
    count (3,001) that leaves the last warp's groups partly past the end."""
    rng = np.random.default_rng(n)
    if kind == "tri":
        items = rng.uniform(0, 10, (n, 9)).astype(np.float32)
    elif kind == "point":
        items = workloads.point_cloud("surface", n, 3) if n > 100 else rng.uniform(0, 10, (n, 3)).astype(np.float32)
    else:
        items = workloads.gaussians(n, 0.05, 1.0, 5)
        items[:, :3] *= 0.1
    tree = capi.DeviceTree(kind, items)
    lo = np.asarray(items).reshape(n, -1)[:, :3].min(0) - 1
    hi = np.asarray(items).reshape(n, -1)[:, :3].max(0) + 1
    q = _dev(workloads.uniform_points(3_001, lo, hi, 7, 13))
    r = float(np.linalg.norm(hi - lo)) * 0.05
    o0, k0 = tree.radius(q, r, 0)
    c0 = tree.closest(q, 0)
    knn0 = {k: tree.knn(q, k, 0) for k in (1, 3, 8, 16)}
    for split in (capi.QK_TUNE_SPLIT, capi.QK_TUNE_SPLIT8, capi.QK_TUNE_SPLIT4):
        for extra in (0, capi.QK_ORDER_MORTON, capi.QK_ORDER_COHERENT):
            f = split | extra
            assert cuda.equal(tree.closest(q, f), c0), (split, extra)
            for k, want in knn0.items():
                assert cuda.equal(tree.knn(q, k, f), want), (split, k, extra)
            o1, k1 = tree.radius(q, r, f)
            assert cuda.equal(o1, o0) and cuda.equal(k1, k0), (split, extra)
        stats = cuda.zeros(4, dtype=cuda.int64, device="cuda")
        tree.knn(q, 8, split, stats=stats)
        assert int(stats[2]) == 0


def _check_small_codes(tree: capi.DeviceTree):
    """Traversal-node words v3.z / v3.w: (first slot << 2) | (leaves - 1) for a child subtree
    of 2..4 leaves on contiguous slots, else 0 (leaf children always 0)."""
    n = tree.n
    nodes = tree.nodes_bytes().view(np.int32).reshape(2 * n - 1, 8)
    bn = tree.host("bnodes", np.int32, (n - 1) * 16).reshape(n - 1, 16)
    depth = tree.host("depth_arr", np.int32, 2 * n - 1)
    first = np.zeros(2 * n - 1, np.int64)
    last = np.zeros(2 * n - 1, np.int64)
    count = np.zeros(2 * n - 1, np.int64)
    first[n - 1:] = last[n - 1:] = np.arange(n)
    count[n - 1:] = 1
    for p in sorted(range(n - 1), key=lambda i: -int(depth[i])):
        l, r = nodes[p, 6], nodes[p, 7]
        first[p] = min(first[l], first[r])
        last[p] = max(last[l], last[r])
        count[p] = count[l] + count[r]
    contiguous = last - first + 1 == count
    small = 0
    for p in range(n - 1):
        for c, word in ((nodes[p, 6], bn[p, 14]), (nodes[p, 7], bn[p, 15])):
            want = 0
            if c < n - 1 and contiguous[c] and 2 <= count[c] <= 4:
                want = (int(first[c]) << 2) | int(count[c] - 1)
                small += 1
            assert int(word) == want, (p, c)
    return small


@pytest.mark.parametrize("kind", ["tri", "point", "gauss"])
@pytest.mark.parametrize("builder", ["lbvh", "sah"])
def test_leaf4_small_subtrees_same_bits(cuda, kind, builder):
    """Child subtrees of 2..4 primitives tested as leaves: same results as the plain binary
    traversal for every query kind, after a refit too (codes depend on the topology only)."""
    items = _items(kind)
    tree = capi.DeviceTree(kind, items, builder=builder)
    assert _check_small_codes(tree) > tree.n // 8
    ref = oracle.LBVH(kind, items)
    qh = _queries(items, kind, 3_001, 5)
    q = _dev(qh)
    lo, hi = qh.min(0), qh.max(0)
    radii = [float(np.linalg.norm(hi - lo)) * f for f in (0.04, 0.2)]
    rays = _dev(_random_rays(lo, hi, 20_001, 6)) if kind == "tri" else None

    def same(t):
        for extra in (0, capi.QK_ORDER_MORTON):
            f = capi.QK_TUNE_LEAF4 | extra
            assert cuda.equal(t.closest(q, f), t.closest(q, 0)), extra
            for k in (1, 8, 16):
                assert cuda.equal(t.knn(q, k, f), t.knn(q, k, 0)), (k, extra)
            # the wide radius reaches leaves whose own box fails the radius although their
            # primitive's computed distance passes it (Gaussians): leaf4 must skip them too
            for r in radii:
                o1, k1 = t.radius(q, r, f)
                o0, k0 = t.radius(q, r, 0)
                assert cuda.equal(o1, o0) and cuda.equal(k1, k0), r
            if rays is not None:
                for tune in (0, capi.QK_TUNE_HIGH_OCC):
                    want, want_ids = t.raycast_ids(rays, extra)
                    got, got_ids = t.raycast_ids(rays, f | tune)
                    assert cuda.equal(got, want) and cuda.equal(got_ids, want_ids)

    same(tree)
    got = tree.closest(q, capi.QK_TUNE_LEAF4).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ref.closest(qh))
    moved = items.copy()
    moved[:, :3] += np.random.default_rng(9).normal(0, 0.05, (len(items), 3)).astype(np.float32)
    tree.refit(moved)
    _check_small_codes(tree)
    same(tree)
    ref.refit(moved)
    got = tree.knn(q, 8, capi.QK_TUNE_LEAF4).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ref.knn(qh, 8))


@pytest.mark.parametrize("n", [2, 3, 4, 5, 9])
def test_leaf4_tiny_trees(cuda, n):
    rng = np.random.default_rng(n)
    pts = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    tree = capi.DeviceTree("point", pts)
    _check_small_codes(tree)
    q = _dev(rng.uniform(-0.5, 1.5, (257, 3)).astype(np.float32))
    f = capi.QK_TUNE_LEAF4
    assert cuda.equal(tree.closest(q, f), tree.closest(q, 0))
    assert cuda.equal(tree.knn(q, min(n, 4), f), tree.knn(q, min(n, 4), 0))
    o1, k1 = tree.radius(q, 0.5, f)
    o0, k0 = tree.radius(q, 0.5, 0)
    assert cuda.equal(o1, o0) and cuda.equal(k1, k0)


def _slot_ranges(nodes: np.ndarray, n: int, depth: np.ndarray):
    """(first slot, leaf count) of every node's subtree, children before parents."""
    first = np.zeros(2 * n - 1, np.int64)
    count = np.zeros(2 * n - 1, np.int64)
    first[n - 1:] = np.arange(n)
    count[n - 1:] = 1
    for p in sorted(range(n - 1), key=lambda i: -int(depth[i])):
        l, r = nodes[p, 6], nodes[p, 7]
        first[p] = min(first[l], first[r])
        count[p] = count[l] + count[r]
    return first, count


@pytest.mark.parametrize("kind", ["tri", "point", "gauss"])
def test_sah4_tree_and_wide_leaf4(cuda, kind):
    """QK_BUILD_SAH4: the SAH decisions stop at ranges of at most 4 primitives, which are split
    by count (left half first).  Every node above them is the binned SAH tree's own node, byte
    for byte, and each range holds the SAH tree's primitives.  qk_wide_build_leaf4 then
    collapses those ranges into single slots: bytes equal the oracle's collapse of the same
    tree, fewer nodes than the plain collapse, every query result equal to the oracle's
    (binary, leaf4, wide; input, Morton and coherent order), and the same after a refit, which
    re-emits the form."""
    items = _items(kind)
    tree = capi.DeviceTree(kind, items, builder="sah4")
    assert tree.validate() == [0] * 8
    again = capi.DeviceTree(kind, items, builder="sah4")
    assert again.nodes_bytes().tobytes() == tree.nodes_bytes().tobytes(), "not deterministic"
    sah = capi.DeviceTree(kind, items, builder="sah")
    n = tree.n
    nodes4 = tree.nodes_bytes().view(np.int32).reshape(2 * n - 1, 8)
    nodes1 = sah.nodes_bytes().view(np.int32).reshape(2 * n - 1, 8)
    depth4 = tree.host("depth_arr", np.int32, 2 * n - 1)
    first4, cnt4 = _slot_ranges(nodes4, n, depth4)
    _, cnt1 = _slot_ranges(nodes1, n, sah.host("depth_arr", np.int32, 2 * n - 1))
    big = np.nonzero(cnt4[: n - 1] > 4)[0]
    assert np.array_equal(big, np.nonzero(cnt1[: n - 1] > 4)[0])
    assert np.array_equal(nodes4[big], nodes1[big])
    parent = tree.host("parent", np.int32, 2 * n - 1)
    ids4, ids1 = tree.host("prim_ids", np.int32, n), sah.host("prim_ids", np.int32, n)
    ranges = 0
    for p in range(n - 1):
        m = int(cnt4[p])
        if m > 4:
            continue
        l, r = nodes4[p, 6], nodes4[p, 7]
        assert cnt4[l] == m // 2 and cnt4[r] == m - m // 2, (p, m)
        if p == 0 or cnt4[parent[p]] > 4:  # a whole leaf range
            f = int(first4[p])
            assert np.array_equal(np.sort(ids4[f:f + m]), np.sort(ids1[f:f + m])), p
            ranges += 1
    assert ranges > n // 8
    assert _check_small_codes(tree) >= ranges

    plain = tree.build_wide()
    ref = oracle.LBVH(kind, items)
    qh = _queries(items, kind, 3_001, 5)
    q = _dev(qh)
    want_c, want_k = ref.closest(qh), ref.knn(qh, 8)
    r = 3.0 if kind != "gauss" else 1.0
    want_off, want_keys = ref.radius(qh, r)
    lo, hi = qh.min(0), qh.max(0)
    rays_h = _random_rays(lo, hi, 20_001, 6) if kind == "tri" else None
    want_r = ref.raycast(rays_h) if kind == "tri" else None

    def same(t):
        for flags in FLAG_SETS + [capi.QK_TUNE_LEAF4, capi.QK_TUNE_LEAF4 | capi.QK_ORDER_MORTON]:
            assert np.array_equal(t.closest(q, flags).cpu().numpy().view(np.uint32), want_c), flags
            assert np.array_equal(t.knn(q, 8, flags).cpu().numpy().view(np.uint32), want_k), flags
            off, keys = t.radius(q, r, flags)
            assert np.array_equal(off.cpu().numpy().astype(np.int64), want_off), flags
            assert np.array_equal(keys.cpu().numpy().view(np.uint64), want_keys), flags
            if rays_h is not None:
                got = t.raycast(_dev(rays_h), flags).cpu().numpy().view(np.uint64)
                assert np.array_equal(got, want_r), flags

    same(tree)  # plain 4-wide form
    count = tree.build_wide(leaf4=True)
    assert tree.t.wide_leaf == 4
    assert count < 0.6 * plain, (count, plain)
    wide, wide_id = oracle.wide_collapse_leaf4(tree.nodes_bytes().view(oracle.NODE_DTYPE),
                                               depth4, n)
    assert count == len(wide) // 4
    assert tree.arrays["wide"].cpu().numpy()[: count * 128].tobytes() == wide.tobytes()
    assert tree.validate() == [0] * 8
    same(tree)  # leaf-size-4 form
    moved = items.copy()
    moved[:, :3] += np.random.default_rng(3).normal(0, 0.05, (len(items), 3)).astype(np.float32)
    tree.refit(moved)
    assert tree.validate() == [0] * 8  # the wide nodes were re-emitted in the leaf4 form
    ref.refit(moved)
    want_c, want_k = ref.closest(qh), ref.knn(qh, 8)
    want_off, want_keys = ref.radius(qh, r)
    want_r = ref.raycast(rays_h) if kind == "tri" else None
    same(tree)


@pytest.mark.parametrize("n", [2, 3, 4, 5, 6, 9, 33, 257])
def test_sah4_tiny_trees(cuda, n):
    """Leaf-size-4 SAH trees small enough that the root, or most of the tree, is one leaf
    range, with the leaf-range 4-wide layer: every query kind on binary, leaf4 and wide
    traversal equals the oracle's."""
    rng = np.random.default_rng(100 + n)
    pts = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    tree = capi.DeviceTree("point", pts, builder="sah4")
    assert tree.validate() == [0] * 8
    tree.build_wide(leaf4=True)
    assert tree.validate() == [0] * 8
    ref = oracle.LBVH("point", pts)
    qh = rng.uniform(-0.5, 1.5, (513, 3)).astype(np.float32)
    q = _dev(qh)
    k = min(n, 4)
    for f in (0, capi.QK_TUNE_LEAF4, capi.QK_WIDE, capi.QK_WIDE | capi.QK_ORDER_MORTON,
              capi.QK_TUNE_SPLIT4):
        assert np.array_equal(tree.closest(q, f).cpu().numpy().view(np.uint32), ref.closest(qh)), f
        assert np.array_equal(tree.knn(q, k, f).cpu().numpy().view(np.uint32), ref.knn(qh, k)), f
        off, keys = tree.radius(q, 0.4, f)
        woff, wkeys = ref.radius(qh, 0.4)
        assert np.array_equal(off.cpu().numpy().astype(np.int64), woff), f
        assert np.array_equal(keys.cpu().numpy().view(np.uint64), wkeys), f


def test_split_knn_sphere_matches_oracle(cuda):
    pts = workloads.point_cloud("surface", 100_000, 2)
    q = workloads.uniform_points(2_000, pts.min(0), pts.max(0), 2, 13)
    tree = capi.DeviceTree("point", pts)
    ref = oracle.LBVH("point", pts)
    got = tree.knn(_dev(q), 8, capi.QK_TUNE_SPLIT).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ref.knn(q, 8))
    got = tree.closest(_dev(q), capi.QK_TUNE_SPLIT).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ref.closest(q))


@pytest.mark.parametrize("kind", ["tri", "point", "gauss"])
def test_radius_stash_same_csr(cuda, kind):
    """Radius with the count pass's 16-key stash: the same CSR as the two-traversal path, with
    segments below, at and above the stash size (and empty ones)."""
    items = _items(kind)
    tree = capi.DeviceTree(kind, items)
    q = _queries(items, kind, 4_001, 31)
    dq = _dev(q)
    lo, hi = q.min(0), q.max(0)
    seen = set()
    for frac in (0.002, 0.03, 0.08, 0.2):
        r = float(np.linalg.norm(hi - lo)) * frac
        o0, k0 = tree.radius(dq, r, 0)
        sizes = np.diff(o0.cpu().numpy())
        seen |= {0 if z == 0 else (1 if z <= 16 else 2) for z in np.unique(sizes)}
        for f in (capi.QK_TUNE_STASH, capi.QK_TUNE_STASH | capi.QK_ORDER_MORTON,
                  capi.QK_TUNE_STASH | capi.QK_TUNE_LEAF4):
            o1, k1 = tree.radius(dq, r, f)
            assert cuda.equal(o1, o0) and cuda.equal(k1, k0), (frac, f)
    assert seen == {0, 1, 2}  # empty segments, segments within the stash and beyond it


def test_radius_segment_sizes_all_sort_paths(cuda):
    """Segments of 0..32 keys (warp registers), 33..1024 (one warp, 32 E keys in registers
    for E = 2, 4, 8, 16, 32: every class occurs), 1025..4096 (block shared memory) and more
    (block, global memory) all come out sorted as the oracle's."""
    rng = np.random.default_rng(21)
    pts = rng.uniform(0, 4, (60_000, 3)).astype(np.float32)
    q = rng.uniform(0.5, 3.5, (400, 3)).astype(np.float32)
    tree = capi.DeviceTree("point", pts)
    ref = oracle.LBVH("point", pts)
    dq = _dev(q)
    classes = set()
    for r in (0.15, 0.25, 0.3, 0.4, 0.55, 0.75, 1.1):
        want_off, want_keys = ref.radius(q, r)
        sizes = np.diff(want_off)
        for flags in (0, capi.QK_TUNE_SPLIT, capi.QK_ORDER_MORTON, capi.QK_TUNE_STASH,
                      capi.QK_TUNE_STASH | capi.QK_ORDER_MORTON):
            off, keys = tree.radius(dq, r, flags)
            assert np.array_equal(off.cpu().numpy().astype(np.int64), want_off)
            assert np.array_equal(keys.cpu().numpy().view(np.uint64), want_keys), (r, flags)
        medium = sizes[(sizes > 32) & (sizes <= 1024)]
        classes |= {int(np.ceil(np.log2(m / 32))) for m in medium}
        if r == 1.1:
            assert sizes.max() > 4096
        if r == 0.75:
            assert ((sizes > 1024) & (sizes <= 4096)).any()
    assert classes == {1, 2, 3, 4, 5}


def test_point_tail_same_results(cuda):
    """QK_TUNE_TAIL: queries near the centre of a 1M-point spherical shell (the search ball of
    such a point admits most of the shell) pass the traversal budget and are answered by the
    shared brute-force scan, in rounds of 1,024 (1,500 of them make two rounds).  Every result
    equals the plain traversal's bits, and the oracle's; stats[3] counts the scanned queries."""
    pts = workloads.point_cloud("surface", 1_048_576, 5)
    tree = capi.DeviceTree("point", pts)
    rng = np.random.default_rng(9)
    centre = rng.normal(0, 2.0, (1_500, 3)).astype(np.float32)  # heavy: near the centre
    spread = workloads.uniform_points(2_500, pts.min(0), pts.max(0), 5, 13)
    q = np.concatenate([centre, spread]).astype(np.float32)
    dq = _dev(q)
    ref = oracle.LBVH("point", pts)
    want_c = ref.closest(q[::7])
    base_c = tree.closest(dq, 0)
    assert np.array_equal(base_c.cpu().numpy().view(np.uint32)[::7], want_c)
    for f in (capi.QK_TUNE_TAIL, capi.QK_TUNE_TAIL | capi.QK_TUNE_SPLIT,
              capi.QK_TUNE_TAIL | capi.QK_TUNE_SPLIT | capi.QK_ORDER_COHERENT,
              capi.QK_TUNE_TAIL | capi.QK_TUNE_SPLIT8, capi.QK_TUNE_TAIL | capi.QK_ORDER_MORTON):
        stats = cuda.zeros(4, dtype=cuda.int64, device="cuda")
        assert cuda.equal(tree.closest(dq, f, stats=stats), base_c), f
        heavy = int(stats[3].item())
        assert heavy >= 1_000, (f, heavy)  # the centre queries went to the scan
        print(f"flags {f}: {heavy} queries scanned")
    for k in (1, 8, 32):
        base = tree.knn(dq, k, 0)
        if k == 8:
            assert np.array_equal(base.cpu().numpy().view(np.uint32)[::7], ref.knn(q[::7], 8))
        for f in (capi.QK_TUNE_TAIL, capi.QK_TUNE_TAIL | capi.QK_TUNE_SPLIT,
                  capi.QK_TUNE_TAIL | capi.QK_TUNE_SPLIT8, capi.QK_TUNE_TAIL | capi.QK_ORDER_COHERENT):
            assert cuda.equal(tree.knn(dq, k, f), base), (k, f)
    # other kinds ignore the flag
    g = capi.DeviceTree("gauss", workloads.gaussians(20_000, 0.05, 1.0, 2))
    gq = _dev(workloads.uniform_points(2_000, [0, 0, 0], [100, 100, 100], 2, 31))
    assert cuda.equal(g.closest(gq, capi.QK_TUNE_TAIL), g.closest(gq, 0))
