"""Zero-copy CUDA path of the module's classes: device arrays in, torch CUDA tensors out,
the same bits as the host path; torch tensors, __cuda_array_interface__ and DLPack inputs."""
from __future__ import annotations

import time

import numpy as np
import pytest

import quarry

pytestmark = pytest.mark.gpu


class CAI:
    """An array that only offers __cuda_array_interface__ (as CuPy or Numba arrays do)."""

    def __init__(self, t):
        self._t = t
        self.__cuda_array_interface__ = t.__cuda_array_interface__


class DLP:
    """An array that only offers DLPack."""

    def __init__(self, t):
        self._t = t

    def __dlpack__(self, stream=None):
        return self._t.__dlpack__()

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


def _same(host, dev):
    if isinstance(host, tuple):
        assert len(host) == len(dev)
        for h, d in zip(host, dev):
            _same(h, d)
        return
    d = dev.cpu().numpy()
    assert d.dtype == host.dtype or (host.dtype == np.bool_ and d.dtype == np.bool_)
    assert np.array_equal(np.ascontiguousarray(host).view(np.uint8),
                          np.ascontiguousarray(d).view(np.uint8))


def test_scene_device_path_equals_host_path(cuda):
    torch = cuda
    v, i = quarry.demo_mesh("terrain", grid=48)
    s = quarry.Scene(v, i, builder="sah")
    b = s.bounds
    lo, hi = np.array(b["min"], np.float32), np.array(b["max"], np.float32)
    rng = np.random.default_rng(1)
    o = np.column_stack([rng.uniform(lo[0], hi[0], 5000), rng.uniform(lo[1], hi[1], 5000),
                         np.full(5000, hi[2] + 5)]).astype(np.float32)
    d = np.tile(np.array([[0.1, -0.05, -1.0]], np.float32), (5000, 1))
    q = (lo + (hi - lo) * rng.random((3000, 3))).astype(np.float32)
    od, dd, qd = (torch.from_numpy(x).cuda() for x in (o, d, q))
    for order in ("input", "morton", "direction"):
        for wide in (False, True):
            _same(s.raycast(o, d, order=order, wide=wide), s.raycast(od, dd, order=order, wide=wide))
    _same(s.raycast(o, d, 40.0), s.raycast(od, dd, 40.0))
    _same(s.closest(q, wide=True), s.closest(qd, wide=True))
    _same(s.knn(q, 7, order="morton"), s.knn(qd, 7, order="morton"))
    _same(s.radius(q, 2.5), s.radius(qd, 2.5))
    # other device array protocols, keyword arguments
    _same(s.closest(q), s.closest(CAI(qd)))
    _same(s.closest(q), s.closest(points=DLP(qd)))
    # results stay on the device
    hit, t = s.raycast(od, dd)
    assert hit.is_cuda and t.is_cuda and t.dtype == torch.float32


@pytest.mark.parametrize("kind", ["point", "gauss"])
def test_clouds_device_path_equals_host_path(cuda, kind):
    torch = cuda
    rng = np.random.default_rng(2)
    if kind == "point":
        pts = rng.uniform(0, 10, (20_000, 3)).astype(np.float32)
        c = quarry.PointCloud(pts)
        lo, hi = pts.min(0), pts.max(0)
    else:
        m, r, sc = quarry.demo_gaussians("sheet", 5000, seed=3)
        c = quarry.GaussianCloud(m, r, sc)
        lo, hi = m.min(0), m.max(0)
    q = (lo + (hi - lo) * rng.random((2000, 3))).astype(np.float32)
    qd = torch.from_numpy(q).cuda()
    for order in ("input", "morton"):
        _same(c.closest(q, order=order), c.closest(qd, order=order))
        _same(c.knn(q, 5, order=order, wide=True), c.knn(qd, 5, order=order, wide=True))
        _same(c.radius(q, 0.4, order=order), c.radius(qd, 0.4, order=order))


def test_device_path_validation_and_overhead(cuda):
    torch = cuda
    pts = np.random.default_rng(3).uniform(0, 1, (50_000, 3)).astype(np.float32)
    c = quarry.PointCloud(pts)
    with pytest.raises(ValueError):
        c.closest(torch.zeros((10, 2), device="cuda"))
    with pytest.raises(ValueError):
        c.knn(torch.zeros((10, 3), device="cuda"), 40)
    q = np.random.default_rng(4).uniform(0, 1, (1000, 3)).astype(np.float32)
    qd = torch.from_numpy(q).cuda()
    for _ in range(5):
        c.closest(q)
        c.closest(qd)
    torch.cuda.synchronize()
    n = 50
    t0 = time.perf_counter()
    for _ in range(n):
        c.closest(q)
    host_us = (time.perf_counter() - t0) / n * 1e6
    t0 = time.perf_counter()
    for _ in range(n):
        c.closest(qd)
    torch.cuda.synchronize()
    dev_us = (time.perf_counter() - t0) / n * 1e6
    print(f"closest of 1,000 points per call: host arrays {host_us:.0f} us, device arrays "
          f"{dev_us:.0f} us")
