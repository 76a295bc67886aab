"""QRYD / QRCD input dumps: byte layout of quarry's writers and round trips (CPU)."""
from __future__ import annotations

import struct

import numpy as np
import pytest

from quarry import dumps, workloads


def test_qryd_bytes_match_the_reference_writer(tmp_path):
    # dumpQueryInput (bench/gpu_query_bench.cpp:232-259): uint32 0x44595251, version 1,
    # uint64 nTris, uint64 nPoints, 9 floats per triangle, 3 per point, little-endian
    tris = np.arange(18, dtype=np.float32).reshape(2, 9) * 0.5
    pts = np.array([[1.0, -2.0, 3.5]], np.float32)
    p = tmp_path / "q.bin"
    dumps.write_qryd(p, tris, pts)
    want = (struct.pack("<IIQQ", 0x44595251, 1, 2, 1) + tris.astype("<f4").tobytes()
            + pts.astype("<f4").tobytes())
    assert p.read_bytes() == want
    assert p.read_bytes()[:4] == b"QRYD"
    t2, p2 = dumps.read_qryd(p)
    assert np.array_equal(t2, tris) and np.array_equal(p2, pts)


def test_qrcd_bytes_match_the_reference_writer(tmp_path):
    # dumpInputs (bench/gpu_cloud_bench.cpp:323-343): "QRCD", uint32 version 1, uint64 np,
    # uint64 nq, float3 points then float3 queries
    pts = workloads.point_cloud("volume", 100, 3)
    q = workloads.uniform_points(7, [0, 0, 0], [1, 1, 1], 3, 13)
    p = tmp_path / "c.bin"
    dumps.write_qrcd(p, pts, q)
    want = b"QRCD" + struct.pack("<IQQ", 1, 100, 7) + pts.tobytes() + q.tobytes()
    assert p.read_bytes() == want
    a, b = dumps.read_qrcd(p)
    assert np.array_equal(a, pts) and np.array_equal(b, q)


def test_bad_files_are_rejected(tmp_path):
    p = tmp_path / "x.bin"
    dumps.write_qrcd(p, np.zeros((3, 3), np.float32), np.zeros((2, 3), np.float32))
    with pytest.raises(ValueError, match="magic"):
        dumps.read_qryd(p)
    data = p.read_bytes()
    (tmp_path / "t.bin").write_bytes(data[:-4])
    with pytest.raises(ValueError, match="bytes"):
        dumps.read_qrcd(tmp_path / "t.bin")
    (tmp_path / "v.bin").write_bytes(data[:4] + struct.pack("<I", 2) + data[8:])
    with pytest.raises(ValueError, match="version"):
        dumps.read_qrcd(tmp_path / "v.bin")
    (tmp_path / "h.bin").write_bytes(data[:10])
    with pytest.raises(ValueError, match="header"):
        dumps.read_qrcd(tmp_path / "h.bin")
