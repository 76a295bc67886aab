"""The oracle's 4-wide collapse in the leaf-size-4 form (oracle/quarry_oracle.c,
qo_wide_collapse_leaf4), checked on its own before it checks the engine.

Walking the wide nodes from the root must reach every leaf slot exactly once, in leaf ranges
of at most four contiguous slots; every slot's box must hold the boxes of the leaves under it
(and equal the leaf box for a single leaf); empty slots stay empty; and the form needs fewer
nodes than quarry's collapse of the same tree.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from quarry import workloads

EMPTY = np.iinfo(np.int32).min


def _walk(wide: np.ndarray, nodes: np.ndarray, n: int) -> np.ndarray:
    seen = np.zeros(n, np.int32)
    leaf_lo = nodes["mn"][n - 1:]
    leaf_hi = nodes["mx"][n - 1:]
    stack = [0]
    visited = 0
    while stack:
        w = stack.pop()
        visited += 1
        assert visited <= len(wide) // 4, "a wide node is reached twice"
        for s in range(4):
            e = wide[4 * w + s]
            c = int(e["child"])
            if c == EMPTY:
                assert int(e["pad"]) == 0
                assert np.all(e["mn"] == np.inf) and np.all(e["mx"] == -np.inf)
                continue
            if c < 0:
                first, cnt = -c - 1, int(e["pad"])
                assert 1 <= cnt <= 4, cnt
                seen[first:first + cnt] += 1
                lo, hi = leaf_lo[first:first + cnt], leaf_hi[first:first + cnt]
                assert np.all(e["mn"] <= lo) and np.all(e["mx"] >= hi)
                if cnt == 1:
                    assert np.array_equal(e["mn"], lo[0]) and np.array_equal(e["mx"], hi[0])
            else:
                assert int(e["pad"]) == 0
                stack.append(c)
    assert visited == len(wide) // 4, "wide nodes nothing points to"
    return seen


@pytest.mark.parametrize("kind,n", [("point", 2), ("point", 3), ("point", 4), ("point", 5),
                                    ("point", 9), ("point", 1000), ("point", 20_000),
                                    ("gauss", 3000), ("tri", None)])
def test_leaf4_collapse_covers_every_leaf_once(kind, n):
    if kind == "tri":
        items = workloads.terrain(40, 2)
    elif kind == "point":
        items = workloads.point_cloud("volume", n, 3)
    else:
        items = workloads.gaussians(n, 0.05, 1.0, 3)
    ref = oracle.LBVH(kind, items)
    wide4, wide_id4 = ref.wide_leaf4()
    seen = _walk(wide4, ref.nodes, ref.n)
    assert np.all(seen == 1)
    wide, _ = ref.wide()
    assert len(wide4) <= len(wide)
    if ref.n >= 1000:
        assert len(wide4) < 0.7 * len(wide), (len(wide4), len(wide))
    # ranges of two or more leaves carry their count; quarry's form keeps pad at zero
    assert np.any(wide4["pad"] >= 2) == (ref.n >= 3)
    assert np.all(wide["pad"] == 0)


def test_leaf4_collapse_of_noncontiguous_subtrees():
    """A tree whose small subtrees do not cover contiguous slots (as topology edits leave
    them) keeps those subtrees as internal slots: coverage stays exact."""
    pts = workloads.point_cloud("volume", 64, 8)
    ref = oracle.LBVH("point", pts)
    nodes = ref.nodes.copy()
    n = ref.n
    # swap the leaf children of two internal nodes whose children are both leaves
    pairs = [i for i in range(n - 1) if nodes[i]["left"] >= n - 1 and nodes[i]["right"] >= n - 1]
    a, b = pairs[0], pairs[-1]
    nodes[a]["right"], nodes[b]["right"] = nodes[b]["right"], nodes[a]["right"]
    # boxes are not what this checks: give every node the root box
    nodes["mn"][: n - 1] = ref.nodes["mn"][0]
    nodes["mx"][: n - 1] = ref.nodes["mx"][0]
    wide4, _ = oracle.wide_collapse_leaf4(nodes, ref.depth_arr, n)
    seen = np.zeros(n, np.int32)
    stack = [0]
    while stack:
        w = stack.pop()
        for s in range(4):
            e = wide4[4 * w + s]
            c = int(e["child"])
            if c == EMPTY:
                continue
            if c < 0:
                seen[-c - 1:-c - 1 + int(e["pad"])] += 1
            else:
                stack.append(c)
    assert np.all(seen == 1)
