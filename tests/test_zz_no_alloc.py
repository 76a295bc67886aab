"""qk_raycast_noalloc, the ray query that allocates nothing, against qk_raycast.

Callers that cannot allocate device memory while they trace (a host that reserves all of it
up front, code without an allocator) use qk_raycast_noalloc: its scratch is a fixed array in
the library, so it takes no workspace.  This test calls it through the C ABI twice in a row,
on different rays and then on the same rays again, and requires the results to equal
qk_raycast's bit for bit (the tolerance of every ray test here: exact), plus a clear error
for a batch over the 262,144-ray limit.  The file sorts last so a stopping run has already
run every other test; it also passes alone in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from quarry import capi, workloads

pytestmark = pytest.mark.gpu


def _noalloc(tree, rays, flags):
    import torch

    out = torch.empty(rays.shape[0], dtype=torch.int64, device="cuda")
    st = capi.lib().qk_raycast_noalloc(ctypes.byref(tree.t), rays.data_ptr(), rays.shape[0],
                                       out.data_ptr(), flags,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    capi.check(st, "qk_raycast_noalloc")
    return out


def test_noalloc_matches_raycast_on_two_calls(cuda):
    tris = workloads.terrain(96, 2)
    tree = capi.DeviceTree("tri", tris)
    tree.build_wide()
    lo, hi = workloads.bounds_of(tris)
    a = capi.to_device(workloads.down_rays(200_000, float(lo[0]), float(hi[0]), float(lo[1]),
                                           float(hi[1]), 50.0, 3), np.float32)
    b = capi.to_device(workloads.cosine_rays(150_000, float(lo[0]), float(hi[0]), float(lo[1]),
                                             float(hi[1]), 40.0, 4), np.float32)
    # input order (no order scratch), Morton (+ 4-wide), the dynamic-fetch schedule (its work
    # counter is a word of the shared scratch, zeroed by the call) and the coherent order
    for flags in (0, capi.QK_ORDER_MORTON, capi.QK_ORDER_MORTON | capi.QK_WIDE,
                  capi.QK_ORDER_MORTON | capi.QK_TUNE_DYNAMIC,
                  capi.QK_ORDER_COHERENT | capi.QK_TUNE_HIGH_OCC):
        want_a = tree.raycast(a, flags)
        want_b = tree.raycast(b, flags)
        got_a = _noalloc(tree, a, flags)
        got_b = _noalloc(tree, b, flags)  # second call in a row reuses the same scratch
        cuda.cuda.synchronize()
        assert cuda.equal(got_a, want_a)
        assert cuda.equal(got_b, want_b)
        assert cuda.equal(_noalloc(tree, a, flags), want_a)


def test_noalloc_rejects_batches_over_the_limit(cuda):
    tris = workloads.terrain(16, 2)
    tree = capi.DeviceTree("tri", tris)
    rays = cuda.zeros((262_145, 8), dtype=cuda.float32, device="cuda")
    out = cuda.empty(262_145, dtype=cuda.int64, device="cuda")
    st = capi.lib().qk_raycast_noalloc(ctypes.byref(tree.t), rays.data_ptr(), 262_145,
                                       out.data_ptr(), capi.QK_ORDER_MORTON, None)
    assert st == 1
    assert b"at most 262144 rays" in capi.lib().qk_last_error()
