"""The engine (C ABI) against the golden fixtures recorded from quarry's CPU reference."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from quarry import capi

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", ["tri", "city", "point", "gauss"])
@pytest.mark.parametrize("builder", ["lbvh", "sah"])
def test_engine_matches_golden_fixtures(cuda, name, builder):
    g = np.load(GOLDEN / f"{name}.npz")
    kind = "tri" if name in ("tri", "city") else name
    tree = capi.DeviceTree(kind, g["items"], builder=builder)
    tree.build_wide()
    q = capi.to_device(g["queries"], np.float32)
    for flags in (0, capi.QK_ORDER_MORTON | capi.QK_WIDE):
        assert np.array_equal(tree.closest(q, flags).cpu().numpy().view(np.uint32), g["closest"])
        assert np.array_equal(tree.knn(q, 8, flags).cpu().numpy().view(np.uint32), g["knn8"])
        off, keys = tree.radius(q, float(g["radius"]), flags)
        assert np.array_equal(off.cpu().numpy().astype(np.int64), g["radius_offsets"])
        assert np.array_equal(keys.cpu().numpy().view(np.uint64), g["radius_keys"])
        if "rays" in g:
            r = capi.to_device(g["rays"], np.float32)
            assert np.array_equal(tree.raycast(r, flags).cpu().numpy().view(np.uint64),
                                  g["ray_results"])
