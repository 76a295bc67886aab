"""Host-side checks of the C ABI library (no GPU needed): it loads, exports every function
include/quarry_b200.h declares, sizes buffers and rejects bad arguments with status codes."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from quarry import capi

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\**\s+\**(qk_[a-z0-9_]+)\(",
                            text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 20
    lib = capi.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(capi.EXPORTS) | {"qk_status_string", "qk_last_error"}


def test_sizes_and_status_strings():
    L = capi.lib()
    s = capi.QkTreeSizes()
    assert L.qk_tree_bytes(capi.QK_TRI, 1000, ctypes.byref(s)) == 0
    assert s.nodes == 1999 * 32 and s.items == 1000 * 36 and s.bnodes == 999 * 64
    assert s.leaves == 1000 * 48
    assert L.qk_tree_bytes(capi.QK_GAUSS, 10, ctypes.byref(s)) == 0 and s.items == 400
    assert L.qk_tree_bytes(capi.QK_POINT, 1, ctypes.byref(s)) == capi.QK_ERR_INVALID if hasattr(capi, "QK_ERR_INVALID") else 1
    assert L.qk_build_workspace_bytes(capi.QK_TRI, 1 << 20, 0) > 16 << 20
    assert L.qk_query_workspace_bytes(1000, 1) > 0
    assert L.qk_stride_floats(0) == 9 and L.qk_stride_floats(1) == 3 and L.qk_stride_floats(2) == 10
    assert L.qk_status_string(0) == b"ok"


def test_bad_arguments_are_rejected_without_touching_the_device():
    L = capi.lib()
    t = capi.QkTree()
    t.kind = 0
    t.n = 1
    assert L.qk_build(ctypes.byref(t), 0, 0, None, None, 0, None) == 1
    assert b"at least 2" in L.qk_last_error()
    assert L.qk_build(None, 0, 0, None, None, 0, None) == 1
    t.n = 100
    t.kind = 7
    assert L.qk_build(ctypes.byref(t), 0, 0, None, None, 0, None) == 1
    assert L.qk_knn(None, None, 0, 0, 0, None, 0, None, None, 0, None) == 1
    assert L.qk_sort_pairs(None, None, None, None, -1, 8, None, 0, None) == 1


@pytest.mark.parametrize("k,stride", [(0, 1), (33, 40), (4, 3)])
def test_knn_argument_checks(k, stride):
    L = capi.lib()
    t = capi.QkTree()
    t.kind = 1
    t.n = 10
    for name in ("nodes", "items", "prim_ids", "parent", "depth_arr", "bnodes", "leaves",
                 "slot_of", "flags"):
        setattr(t, name, 16)  # never dereferenced: the checks run first
    assert L.qk_knn(ctypes.byref(t), None, 0, k, stride, None, 0, None, None, 0, None) == 1


def test_batch_sizes_and_argument_checks():
    L = capi.lib()
    counts = (ctypes.c_int32 * 3)(1000, 5000, 2)
    a = L.qk_batch_arena_bytes(capi.QK_TRI, counts, 3, 0)
    w = L.qk_batch_arena_bytes(capi.QK_TRI, counts, 3, capi.QK_WIDE)
    # at least the three trees' arrays, and the 4-wide fields only when asked for
    s = capi.QkTreeSizes()
    need = 0
    for n in (1000, 5000, 2):
        L.qk_tree_bytes(capi.QK_TRI, n, ctypes.byref(s))
        need += s.nodes + s.items + s.bnodes + s.leaves
    assert a > need and w > a + (999 + 4999 + 1) * 128
    bad = (ctypes.c_int32 * 2)(1000, 1)
    assert L.qk_batch_arena_bytes(capi.QK_TRI, bad, 2, 0) == 0
    h = ctypes.c_void_p()
    assert L.qk_batch_create(ctypes.byref(h), capi.QK_TRI, bad, 2, 16, 256, 1 << 30, 0, None) == 1
    assert b"at least 2" in L.qk_last_error()
    # unaligned arena, unknown flags, too-small arena: rejected before any device call
    assert L.qk_batch_create(ctypes.byref(h), capi.QK_TRI, counts, 3, 16, 260, a, 0, None) == 1
    assert L.qk_batch_create(ctypes.byref(h), capi.QK_TRI, counts, 3, 16, 256, a, 8, None) == 1
    assert L.qk_batch_create(ctypes.byref(h), capi.QK_TRI, counts, 3, 16, 256, a - 1, 0, None) == 3
    assert not h.value
    assert L.qk_batch_query(None, None, None, 0, None) == 1
    assert L.qk_batch_plan_status(None, None, None, None) == 1


def test_batch_workload_sizes_are_seeded():
    from quarry import workloads

    sizes = [workloads.batch_scene_sizes(i, (1_000, 500_000), (1_000, 100_000)) for i in range(256)]
    assert sizes == [workloads.batch_scene_sizes(i, (1_000, 500_000), (1_000, 100_000))
                     for i in range(256)]
    n = [s[0] for s in sizes]
    q = [s[1] for s in sizes]
    assert min(n) >= 1_000 and max(n) <= 500_000 and min(q) >= 1_000 and max(q) <= 100_000
    # log-uniform: about half the draws below the geometric midpoint
    assert 80 < sum(x < (1_000 * 500_000) ** 0.5 for x in n) < 176
    cfg = workloads.batch_config(terrains=2, clouds=2, tri_range=(1_000, 4_000),
                                 point_range=(4_000, 8_000), query_range=(30, 90))
    for sc in cfg.terrains + cfg.clouds:
        q3 = sc.closest.shape[0] + sc.knn.shape[0] + sc.radius.shape[0]
        assert sc.closest.shape[0] == sc.knn.shape[0] == q3 // 3
        assert sc.r > 0
        assert sc.rays.shape[0] == (q3 if sc.kind == "tri" else 0)


def test_header_constants_match_python():
    """Every QK_* value the header defines equals the Python module's constant of that name."""
    import re

    text = (Path(__file__).resolve().parents[1] / "include" / "quarry_b200.h").read_text()
    defs = {m.group(1): int(m.group(2)) for m in
            re.finditer(r"^#define (QK_\w+) (\d+)u?\b", text, re.M)}
    assert defs["QK_ORDER_COHERENT"] == 8
    shared = [k for k in defs if hasattr(capi, k)]
    assert len(shared) >= 15
    for k in shared:
        assert getattr(capi, k) == defs[k], k
