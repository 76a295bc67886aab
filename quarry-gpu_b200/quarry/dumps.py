"""quarry's binary input dumps, so other engines can be fed byte-identical inputs.

Both formats are little-endian: a 4-byte magic, a uint32 version (1), two uint64 counts,
then float32 records.

  QRYD (bench/gpu_query_bench.cpp:232-259): "QRYD", version, n_tris, n_points,
        n_tris x 9 floats (a.xyz b.xyz c.xyz), n_points x 3 floats
  QRCD (bench/gpu_cloud_bench.cpp:323-343): "QRCD", version, n_points, n_queries,
        n_points x 3 floats, n_queries x 3 floats
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

_HEADER = struct.Struct("<4sIQQ")
VERSION = 1


def _write(path, magic: bytes, a: np.ndarray, b: np.ndarray, wa: int, wb: int) -> None:
    a = np.ascontiguousarray(a, dtype="<f4").reshape(-1, wa)
    b = np.ascontiguousarray(b, dtype="<f4").reshape(-1, wb)
    with open(path, "wb") as f:
        f.write(_HEADER.pack(magic, VERSION, a.shape[0], b.shape[0]))
        f.write(a.tobytes())
        f.write(b.tobytes())


def _read(path, magic: bytes, wa: int, wb: int) -> tuple[np.ndarray, np.ndarray]:
    data = Path(path).read_bytes()
    if len(data) < _HEADER.size:
        raise ValueError(f"{path}: shorter than the {_HEADER.size}-byte header")
    m, version, na, nb = _HEADER.unpack_from(data, 0)
    if m != magic:
        raise ValueError(f"{path}: magic {m!r} is not {magic!r}")
    if version != VERSION:
        raise ValueError(f"{path}: version {version} is not {VERSION}")
    need = _HEADER.size + 4 * (na * wa + nb * wb)
    if len(data) != need:
        raise ValueError(f"{path}: {len(data)} bytes, the header describes {need}")
    off = _HEADER.size
    a = np.frombuffer(data, dtype="<f4", count=na * wa, offset=off).reshape(na, wa)
    off += 4 * na * wa
    b = np.frombuffer(data, dtype="<f4", count=nb * wb, offset=off).reshape(nb, wb)
    return a.astype(np.float32), b.astype(np.float32)


def write_qryd(path, tris: np.ndarray, points: np.ndarray) -> None:
    """Triangles (n, 9) and query points (m, 3) as a QRYD file."""
    _write(path, b"QRYD", tris, points, 9, 3)


def read_qryd(path) -> tuple[np.ndarray, np.ndarray]:
    """(triangles (n, 9), points (m, 3)) of a QRYD file."""
    return _read(path, b"QRYD", 9, 3)


def write_qrcd(path, points: np.ndarray, queries: np.ndarray) -> None:
    """A point cloud (n, 3) and query points (m, 3) as a QRCD file."""
    _write(path, b"QRCD", points, queries, 3, 3)


def read_qrcd(path) -> tuple[np.ndarray, np.ndarray]:
    """(points (n, 3), queries (m, 3)) of a QRCD file."""
    return _read(path, b"QRCD", 3, 3)
