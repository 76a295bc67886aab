"""Error statuses of the traversal entry points, exercised without faulting anything.

A tree the engine builds is never deeper than its traversal stacks (the SAH builder halves a
range by count when a split would pass depth 62; a 64-bit-key LBVH cannot pass 62).  A tree
assembled by a caller can be, so this file assembles one on the host: a "comb" of 100
internal nodes whose left child continues the chain and whose right child is a two-leaf
node, every box the same, so each chain node has two children to visit and a depth-first
traversal pushes one entry per level (the reference's stack-overflow case,
bench/gpu_bench.cpp:327-330).  Every child index is checked on the CPU to lie inside the
arrays before anything runs on the GPU.

* With the true depth recorded in the tree, every traversal entry point returns
  QK_ERR_DEPTH before launching anything.
* With a smaller depth recorded (a caller's mistake), the kernels run, stop each traversal
  at the stack limit (every push checks the stack size first; every loop has an iteration
  cap) and report the overflows in the statistics words; the process and the context stay
  usable.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from quarry import capi

pytestmark = pytest.mark.gpu

CHAIN = 100  # internal chain nodes; the tree's depth is CHAIN


def comb_tree():
    """Host arrays of the comb: internal nodes 0..2m-1 (chain i = i, pair node A_i = m + i),
    n = 2m + 1 leaves; A_i holds slots 2i, 2i+1, the last chain node's left child slot 2m.
    Returns (n, canonical nodes (2n-1, 8) f32 view, bnodes (n-1, 16) f32 view, leaves
    (n, 12) f32, tris (n, 9), depth)."""
    m = CHAIN
    n_int = 2 * m
    n = n_int + 1
    lo, hi = (0.0, 0.0, -1.0), (1.0, 1.0, 1.0)
    refs = np.zeros((n_int, 2), np.int32)
    for i in range(m):
        refs[i, 0] = i + 1 if i + 1 < m else ~(2 * m)   # left: the chain continues
        refs[i, 1] = m + i                               # right: the pair node
        refs[m + i, 0] = ~(2 * i)
        refs[m + i, 1] = ~(2 * i + 1)
    # every reference in range: internal ids in [0, n-2], leaf slots in [0, n-1]
    internal = refs[refs >= 0]
    slots = ~refs[refs < 0]
    assert internal.min() >= 0 and internal.max() <= n - 2
    assert slots.min() >= 0 and slots.max() <= n - 1
    assert np.unique(slots).size == n  # every leaf exactly once

    bn = np.zeros((n - 1, 16), np.float32)
    bn[:, 0:3] = lo
    bn[:, 3:6] = hi
    bn[:, 6:9] = lo
    bn[:, 9:12] = hi
    bn.view(np.int32)[:, 12:14] = refs
    nodes = np.zeros((2 * n - 1, 8), np.float32)
    nodes[:, 0:3] = lo
    nodes[:, 3:6] = hi
    nodes.view(np.int32)[: n - 1, 6:8] = refs
    nodes.view(np.int32)[n - 1:, 6:8] = -1
    tris = np.zeros((n, 9), np.float32)
    tris[:, 0:3] = (0.1, 0.1, 0.0)
    tris[:, 3:6] = (0.9, 0.1, 0.0)
    tris[:, 6:9] = (0.1, 0.9, 0.0)
    leaves = np.zeros((n, 12), np.float32)
    leaves[:, 0:3] = tris[:, 0:3]
    leaves[:, 4:7] = tris[:, 3:6]
    leaves[:, 8:11] = tris[:, 6:9]
    leaves.view(np.int32)[:, 3] = np.arange(n)
    return n, nodes, bn, leaves, tris, m


def _tree(cuda, depth):
    n, nodes, bn, leaves, tris, true_depth = comb_tree()
    keep = {}

    def dev(a):
        t = cuda.from_numpy(np.ascontiguousarray(a)).to("cuda")
        keep[id(t)] = t
        return t.data_ptr()

    t = capi.QkTree()
    t.kind = 0
    t.n = n
    t.depth = depth
    t.nodes = dev(nodes)
    t.items = dev(tris)
    t.prim_ids = dev(np.arange(n, dtype=np.int32))
    t.parent = dev(np.full(2 * n - 1, -1, np.int32))
    t.depth_arr = dev(np.zeros(2 * n - 1, np.int32))
    t.bnodes = dev(bn)
    t.leaves = dev(leaves)
    t.slot_of = dev(np.arange(n, dtype=np.int32))
    t.flags = dev(np.zeros(n - 1, np.int32))
    t.wide = None
    t.wide_id = dev(np.zeros(n - 1, np.int32))
    return t, keep, true_depth


def _rays(cuda, count):
    r = np.zeros((count, 8), np.float32)
    r[:, 0] = np.linspace(0.2, 0.3, count)
    r[:, 1] = 0.2
    r[:, 2] = 0.5
    r[:, 5] = -1.0
    r[:, 6] = 1e-6
    r[:, 7] = np.inf
    return cuda.from_numpy(r).to("cuda")


def test_too_deep_tree_is_refused_before_any_launch(cuda):
    t, keep, depth = _tree(cuda, CHAIN)
    assert depth == CHAIN >= 64
    L = capi.lib()
    rays = _rays(cuda, 64)
    out = cuda.empty(64, dtype=cuda.int64, device="cuda")
    pts = cuda.full((64, 3), 0.5, device="cuda")
    res = cuda.empty((64, 2), dtype=cuda.int32, device="cuda")
    knn = cuda.empty((64, 4, 2), dtype=cuda.int32, device="cuda")
    offs = cuda.empty(65, dtype=cuda.int32, device="cuda")
    total = ctypes.c_int64(0)
    ws = cuda.empty(1 << 20, dtype=cuda.uint8, device="cuda")
    wsb = ws.numel()
    calls = {
        "qk_raycast": lambda: L.qk_raycast(ctypes.byref(t), rays.data_ptr(), 64, out.data_ptr(),
                                           0, None, ws.data_ptr(), wsb, None),
        "qk_closest": lambda: L.qk_closest(ctypes.byref(t), pts.data_ptr(), 64, res.data_ptr(), 0,
                                           None, ws.data_ptr(), wsb, None),
        "qk_knn": lambda: L.qk_knn(ctypes.byref(t), pts.data_ptr(), 64, 4, 4, knn.data_ptr(), 0,
                                   None, ws.data_ptr(), wsb, None),
        "qk_radius_count": lambda: L.qk_radius_count(ctypes.byref(t), pts.data_ptr(), 64,
                                                     ctypes.c_float(0.5), offs.data_ptr(),
                                                     ctypes.byref(total), 0, None, ws.data_ptr(),
                                                     wsb, None),
        "qk_raycast_noalloc": lambda: L.qk_raycast_noalloc(ctypes.byref(t), rays.data_ptr(), 64,
                                                           out.data_ptr(), 0, None),
    }
    for name, call in calls.items():
        st = call()
        assert st == 5, (name, st)  # QK_ERR_DEPTH
        assert b"exceeds the traversal stack" in L.qk_last_error(), name
    cuda.cuda.synchronize()


def test_stack_overflow_is_counted_not_faulted(cuda):
    # a caller that records too small a depth: the kernels run, stop every traversal at the
    # stack limit and count it; results of stopped traversals are not meaningful
    t, keep, _ = _tree(cuda, 10)
    count = 256
    rays = _rays(cuda, count)
    out = cuda.empty(count, dtype=cuda.int64, device="cuda")
    stats = cuda.zeros(4, dtype=cuda.int64, device="cuda")
    ws = cuda.empty(1 << 20, dtype=cuda.uint8, device="cuda")
    L = capi.lib()
    st = L.qk_raycast(ctypes.byref(t), rays.data_ptr(), count, out.data_ptr(), 0,
                      stats.data_ptr(), ws.data_ptr(), ws.numel(), None)
    capi.check(st, "qk_raycast")
    cuda.cuda.synchronize()
    s = stats.cpu().numpy()
    assert s[2] == count, s  # every ray stopped at the stack limit
    pts = cuda.tensor(np.tile([[0.5, 0.5, 0.5]], (count, 1)).astype(np.float32), device="cuda")
    res = cuda.empty((count, 2), dtype=cuda.int32, device="cuda")
    stats.zero_()
    st = L.qk_closest(ctypes.byref(t), pts.data_ptr(), count, res.data_ptr(), 0,
                      stats.data_ptr(), ws.data_ptr(), ws.numel(), None)
    capi.check(st, "qk_closest")
    cuda.cuda.synchronize()
    assert stats.cpu().numpy()[2] == count
    # the context is still usable: an ordinary tree answers as before
    from quarry import workloads

    tris = workloads.terrain(16, 1)
    good = capi.DeviceTree("tri", tris)
    r2 = capi.to_device(workloads.down_rays(1000, 0.0, 16.0, 0.0, 16.0, 100.0, 1), np.float32)
    hits = good.raycast(r2).cpu().numpy()
    assert ((hits >> 32) != 0).all()
