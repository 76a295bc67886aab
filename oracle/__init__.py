"""ctypes front end of the oracle.  TEST INFRASTRUCTURE ONLY.

Loads the C restatement (oracle/_build/liboracle.so, built from quarry_oracle.c by
oracle/Makefile) and, when present, quarry's own CPU reference compiled from its sources
(oracle/_ref/libquarry_ref.so).  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs import this module; the engine never does.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
REF_PATH = HERE / "_ref" / "libquarry_ref.so"
REFERENCE_SRC = Path("/root/reference")

KIND = {"tri": 0, "point": 1, "gauss": 2}
STRIDE = {0: 9, 1: 3, 2: 10}
NODE_DTYPE = np.dtype([("mn", "<f4", 3), ("mx", "<f4", 3), ("left", "<i4"), ("right", "<i4")])
WIDE_DTYPE = np.dtype([("mn", "<f4", 3), ("mx", "<f4", 3), ("child", "<i4"), ("pad", "<i4")])

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_F = ctypes.c_float
_U64 = ctypes.c_uint64
_D = ctypes.c_double


def build(reference: bool = True) -> None:
    """Compile the restatement, and the reference shim when the reference sources exist."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    if reference and REFERENCE_SRC.is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REFERENCE_SRC}"], check=True)
        # quarry's own callers against the engine's header and library (drop-in check); they
        # link libquarry_b200.so, so the engine is built first
        engine = HERE.parent / "quarry-gpu_b200" / "quarry" / "libquarry_b200.so"
        if engine.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "callers", f"REF={REFERENCE_SRC}"],
                           check=True)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_P)


def _sig(lib, name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build(reference=False)
        L = ctypes.CDLL(str(LIB_PATH))
        _sig(L, "qo_intersect_aabb", _I, [_P, _P, _F, _P])
        _sig(L, "qo_intersect_triangle", _I, [_P, _P, _P])
        _sig(L, "qo_closest_point_dist2", _F, [_P, _P])
        _sig(L, "qo_dist2_aabb", _F, [_P, _P])
        _sig(L, "qo_gaussian_bounds", None, [_P, _P])
        _sig(L, "qo_gaussian_dist2", _F, [_P, _P])
        _sig(L, "qo_prim_dist2", _F, [_I, _P, _P])
        _sig(L, "qo_prim_bounds", None, [_I, _P, _P])
        _sig(L, "qo_lbvh_build", _I, [_I, _P, _I, _P, _P, _P, _P, _P])
        _sig(L, "qo_wide_collapse", _I, [_P, _P, _I, _P, _P])
        _sig(L, "qo_wide_collapse_leaf4", _I, [_P, _P, _I, _P, _P])
        _sig(L, "qo_refit", None, [_I, _P, _P, _I])
        _sig(L, "qo_raycast", None, [_P, _P, _P, _I, _P, _I, _P, _I])
        _sig(L, "qo_closest", None, [_I, _P, _P, _P, _I, _P, _I, _P, _I])
        _sig(L, "qo_knn", None, [_I, _P, _P, _P, _I, _P, _I, _I, _P, _I])
        _sig(L, "qo_radius", _I64, [_I, _P, _P, _P, _I, _P, _I, _F, _P, _P, _P, _I])
        _sig(L, "qo_raycast_brute", None, [_P, _I, _P, _I, _P])
        _sig(L, "qo_closest_brute", None, [_I, _P, _I, _P, _I, _P])
        _sig(L, "qo_knn_brute", None, [_I, _P, _I, _P, _I, _I, _P])
        _sig(L, "qo_ray_hash", _U64, [_P, _I64, _P])
        _sig(L, "qo_closest_hash", _U64, [_P, _I64])
        _sig(L, "qo_knn_hash", _U64, [_P, _I64, _I])
        _sig(L, "qo_radius_hash", _U64, [_P, _P, _I64])
        _sig(L, "qo_bytes_hash", _U64, [_P, ctypes.c_size_t])
        _lib = L
    return _lib


def ref_available() -> bool:
    if REF_PATH.exists():
        return True
    if REFERENCE_SRC.is_dir():
        try:
            build(reference=True)
        except Exception:  # pragma: no cover - reported by the caller
            return False
    return REF_PATH.exists()


def ref():
    """quarry's own CPU reference (oracle/_ref), compiled from its sources."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("oracle/_ref/libquarry_ref.so is not built")
        R = ctypes.CDLL(str(REF_PATH))
        _sig(R, "qr_selftest", _I, [])
        _sig(R, "qr_intersect_triangle", _I, [_P, _P, _P])
        _sig(R, "qr_closest_point_dist2", _F, [_P, _P])
        _sig(R, "qr_gaussian_dist2", _F, [_P, _P])
        _sig(R, "qr_gaussian_bounds", None, [_P, _P])
        _sig(R, "qr_dist2_aabb", _F, [_P, _P])
        _sig(R, "qr_raycast", _D, [_P, _I, _P, _I, _P, _I, _P])
        _sig(R, "qr_raycast_brute", None, [_P, _I, _P, _I, _P])
        _sig(R, "qr_closest", _D, [_I, _P, _I, _P, _I, _P, _I, _P])
        _sig(R, "qr_knn", _D, [_I, _P, _I, _P, _I, _I, _P, _I, _P])
        _sig(R, "qr_radius", _P, [_I, _P, _I, _P, _I, _F, _I, _P])
        _sig(R, "qr_radius_total", _I64, [_P])
        _sig(R, "qr_radius_copy", None, [_P, _P, _P])
        _sig(R, "qr_radius_free", None, [_P])
        _sig(R, "qr_closest_brute", None, [_I, _P, _I, _P, _I, _P])
        _sig(R, "qr_ray_hash", _U64, [_P, _I64, _P])
        _sig(R, "qr_closest_hash", _U64, [_P, _I64])
        _sig(R, "qr_list_hash", _U64, [_P, _P, _I64])
        _sig(R, "qr_scene", _P, [_I, _P, _I, _P, _I, _P, _P, _I, _I, _P, _P, _I, _F, _P, _I, _P,
                                 _I, _P, _P])
        _ref = R
    return _ref


SCENES_PATH = HERE / "_build" / "libqscenes.so"
_scenes = None


def scenes_lib() -> ctypes.CDLL:
    """The engine's workload generators (quarry-gpu_b200/csrc/scenes.c) compiled on their own
    by oracle/Makefile, for CPU-side runs that must not load the engine library; the same
    source and flags as the engine's copy, so the same bytes (tests/test_workloads.py)."""
    global _scenes
    if _scenes is None:
        if not SCENES_PATH.exists():
            build(reference=False)
        _scenes = ctypes.CDLL(str(SCENES_PATH))
    return _scenes


def standalone_workloads():
    """quarry-gpu_b200/quarry/workloads.py loaded as a plain module bound to scenes_lib(): the
    benchmark inputs without importing the quarry package or its libraries."""
    import importlib.util
    import sys

    name = "_qk_workloads_standalone"
    if name in sys.modules:
        return sys.modules[name]
    path = HERE.parent / "quarry-gpu_b200" / "quarry" / "workloads.py"
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    mod.bind(scenes_lib())
    return mod


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


# --------------------------------------------------------------------------------------
# the C restatement
# --------------------------------------------------------------------------------------
class LBVH:
    """LBVH built by the restatement of src/gpu/lbvh.cu (bit-identical node array)."""

    def __init__(self, kind: str, items: np.ndarray):
        self.kind = KIND[kind]
        items = _f32(items).reshape(-1, STRIDE[self.kind])
        self.n = n = items.shape[0]
        if n < 2:
            raise ValueError("at least 2 primitives are required")
        self.nodes = np.zeros(2 * n - 1, dtype=NODE_DTYPE)
        self.sorted = np.zeros_like(items)
        self.prim_ids = np.zeros(n, dtype=np.int32)
        self.parent = np.zeros(2 * n - 1, dtype=np.int32)
        self.depth_arr = np.zeros(2 * n - 1, dtype=np.int32)
        self.depth = lib().qo_lbvh_build(self.kind, _ptr(items), n, _ptr(self.nodes),
                                         _ptr(self.sorted), _ptr(self.prim_ids),
                                         _ptr(self.parent), _ptr(self.depth_arr))

    def tree_hash(self) -> int:
        return lib().qo_bytes_hash(_ptr(self.nodes), self.nodes.nbytes)

    def wide(self):
        n = self.n
        wide_id = np.zeros(n - 1, dtype=np.int32)
        wide = np.zeros((n - 1) * 4, dtype=WIDE_DTYPE)
        count = lib().qo_wide_collapse(_ptr(self.nodes), _ptr(self.depth_arr), n, _ptr(wide_id),
                                       _ptr(wide))
        return wide[: 4 * count].copy(), wide_id

    def wide_leaf4(self):
        return wide_collapse_leaf4(self.nodes, self.depth_arr, self.n)

    def refit(self, items: np.ndarray) -> None:
        """Topology-frozen refit with scene-ordered items (same count)."""
        items = _f32(items).reshape(-1, STRIDE[self.kind])
        self.sorted = np.ascontiguousarray(items[self.prim_ids])
        lib().qo_refit(self.kind, _ptr(self.nodes), _ptr(self.sorted), self.n)

    def raycast(self, rays: np.ndarray, threads: int = 0) -> np.ndarray:
        rays = _f32(rays).reshape(-1, 8)
        out = np.zeros(rays.shape[0], dtype=np.uint64)
        lib().qo_raycast(_ptr(self.nodes), _ptr(self.sorted), _ptr(self.prim_ids), self.n,
                         _ptr(rays), rays.shape[0], _ptr(out), threads)
        return out

    def closest(self, q: np.ndarray, threads: int = 0) -> np.ndarray:
        q = _f32(q).reshape(-1, 3)
        out = np.zeros((q.shape[0], 2), dtype=np.uint32)
        lib().qo_closest(self.kind, _ptr(self.nodes), _ptr(self.sorted), _ptr(self.prim_ids),
                         self.n, _ptr(q), q.shape[0], _ptr(out), threads)
        return out

    def knn(self, q: np.ndarray, k: int, threads: int = 0) -> np.ndarray:
        q = _f32(q).reshape(-1, 3)
        out = np.zeros((q.shape[0], k, 2), dtype=np.uint32)
        lib().qo_knn(self.kind, _ptr(self.nodes), _ptr(self.sorted), _ptr(self.prim_ids),
                     self.n, _ptr(q), q.shape[0], k, _ptr(out), threads)
        return out

    def radius(self, q: np.ndarray, r: float, threads: int = 0):
        q = _f32(q).reshape(-1, 3)
        nq = q.shape[0]
        counts = np.zeros(nq, dtype=np.int32)
        lib().qo_radius(self.kind, _ptr(self.nodes), _ptr(self.sorted), _ptr(self.prim_ids),
                        self.n, _ptr(q), nq, r, _ptr(counts), None, None, threads)
        offsets = np.zeros(nq + 1, dtype=np.int64)
        np.cumsum(counts, out=offsets[1:])
        keys = np.zeros(int(offsets[-1]), dtype=np.uint64)
        lib().qo_radius(self.kind, _ptr(self.nodes), _ptr(self.sorted), _ptr(self.prim_ids),
                        self.n, _ptr(q), nq, r, _ptr(counts), _ptr(offsets), _ptr(keys), threads)
        return offsets, keys


def wide_collapse_leaf4(nodes: np.ndarray, depth: np.ndarray, n: int):
    """Leaf-size-4 4-wide collapse (qo_wide_collapse_leaf4) of any tree in the canonical node
    format (2n-1 NODE_DTYPE entries, root 0) with its node depths: (wide nodes, wide_id)."""
    nodes = np.ascontiguousarray(nodes, dtype=NODE_DTYPE)
    depth = np.ascontiguousarray(depth, dtype=np.int32)
    wide_id = np.zeros(n - 1, dtype=np.int32)
    wide = np.zeros((n - 1) * 4, dtype=WIDE_DTYPE)
    count = lib().qo_wide_collapse_leaf4(_ptr(nodes), _ptr(depth), n, _ptr(wide_id), _ptr(wide))
    if count < 0:
        raise MemoryError("qo_wide_collapse_leaf4")
    return wide[: 4 * count].copy(), wide_id


def raycast_brute(tris, rays) -> np.ndarray:
    tris = _f32(tris).reshape(-1, 9)
    rays = _f32(rays).reshape(-1, 8)
    out = np.zeros(rays.shape[0], dtype=np.uint64)
    lib().qo_raycast_brute(_ptr(tris), tris.shape[0], _ptr(rays), rays.shape[0], _ptr(out))
    return out


def closest_brute(kind: str, items, q) -> np.ndarray:
    k = KIND[kind]
    items = _f32(items).reshape(-1, STRIDE[k])
    q = _f32(q).reshape(-1, 3)
    out = np.zeros((q.shape[0], 2), dtype=np.uint32)
    lib().qo_closest_brute(k, _ptr(items), items.shape[0], _ptr(q), q.shape[0], _ptr(out))
    return out


def knn_brute(kind: str, items, q, k: int) -> np.ndarray:
    kk = KIND[kind]
    items = _f32(items).reshape(-1, STRIDE[kk])
    q = _f32(q).reshape(-1, 3)
    out = np.zeros((q.shape[0], k, 2), dtype=np.uint32)
    lib().qo_knn_brute(kk, _ptr(items), items.shape[0], _ptr(q), q.shape[0], k, _ptr(out))
    return out


def ray_hash(res: np.ndarray) -> tuple[int, int]:
    res = np.ascontiguousarray(res, dtype=np.uint64)
    hits = ctypes.c_uint64(0)
    h = lib().qo_ray_hash(_ptr(res), res.size, ctypes.byref(hits))
    return h, hits.value


def closest_hash(res2: np.ndarray) -> int:
    res2 = np.ascontiguousarray(res2, dtype=np.uint32).reshape(-1, 2)
    return lib().qo_closest_hash(_ptr(res2), res2.shape[0])


def knn_hash(res2: np.ndarray) -> int:
    res2 = np.ascontiguousarray(res2, dtype=np.uint32)
    nq, k = res2.shape[0], res2.shape[1]
    return lib().qo_knn_hash(_ptr(res2), nq, k)


def radius_hash(offsets: np.ndarray, keys: np.ndarray) -> int:
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    return lib().qo_radius_hash(_ptr(offsets), _ptr(keys), offsets.size - 1)


def bytes_hash(buf: np.ndarray) -> int:
    buf = np.ascontiguousarray(buf)
    return lib().qo_bytes_hash(_ptr(buf), buf.nbytes)


def prim_dist2(kind: str, q, item) -> float:
    q = _f32(q)
    item = _f32(item)
    return lib().qo_prim_dist2(KIND[kind], _ptr(q), _ptr(item))


def prim_bounds(kind: str, item) -> np.ndarray:
    item = _f32(item)
    box = np.zeros(6, dtype=np.float32)
    lib().qo_prim_bounds(KIND[kind], _ptr(item), _ptr(box))
    return box


def intersect_triangle(ray, tri):
    ray = _f32(ray)
    tri = _f32(tri)
    t = ctypes.c_float(0.0)
    ok = lib().qo_intersect_triangle(_ptr(ray), _ptr(tri), ctypes.byref(t))
    return bool(ok), t.value


# --------------------------------------------------------------------------------------
# quarry's own CPU reference (oracle/_ref)
# --------------------------------------------------------------------------------------
class Reference:
    """Thin numpy layer over oracle/_ref/libquarry_ref.so."""

    def __init__(self):
        self.R = ref()

    def selftest(self) -> bool:
        return bool(self.R.qr_selftest())

    def raycast(self, tris, rays, threads: int = 0):
        tris = _f32(tris).reshape(-1, 9)
        rays = _f32(rays).reshape(-1, 8)
        out = np.zeros(rays.shape[0], dtype=np.uint64)
        bms = ctypes.c_double(0.0)
        ms = self.R.qr_raycast(_ptr(tris), tris.shape[0], _ptr(rays), rays.shape[0], _ptr(out),
                               threads, ctypes.byref(bms))
        return out, ms, bms.value

    def raycast_brute(self, tris, rays):
        tris = _f32(tris).reshape(-1, 9)
        rays = _f32(rays).reshape(-1, 8)
        out = np.zeros(rays.shape[0], dtype=np.uint64)
        self.R.qr_raycast_brute(_ptr(tris), tris.shape[0], _ptr(rays), rays.shape[0], _ptr(out))
        return out

    def closest(self, kind: str, items, q, threads: int = 0):
        k = KIND[kind]
        items = _f32(items).reshape(-1, STRIDE[k])
        q = _f32(q).reshape(-1, 3)
        out = np.zeros((q.shape[0], 2), dtype=np.uint32)
        bms = ctypes.c_double(0.0)
        ms = self.R.qr_closest(k, _ptr(items), items.shape[0], _ptr(q), q.shape[0], _ptr(out),
                               threads, ctypes.byref(bms))
        return out, ms, bms.value

    def knn(self, kind: str, items, q, kk: int, threads: int = 0):
        k = KIND[kind]
        items = _f32(items).reshape(-1, STRIDE[k])
        q = _f32(q).reshape(-1, 3)
        out = np.zeros((q.shape[0], kk, 2), dtype=np.uint32)
        bms = ctypes.c_double(0.0)
        ms = self.R.qr_knn(k, _ptr(items), items.shape[0], _ptr(q), q.shape[0], kk, _ptr(out),
                           threads, ctypes.byref(bms))
        return out, ms, bms.value

    def radius(self, kind: str, items, q, r: float, threads: int = 0):
        k = KIND[kind]
        items = _f32(items).reshape(-1, STRIDE[k])
        q = _f32(q).reshape(-1, 3)
        qms = ctypes.c_double(0.0)
        h = self.R.qr_radius(k, _ptr(items), items.shape[0], _ptr(q), q.shape[0], r, threads,
                             ctypes.byref(qms))
        try:
            total = self.R.qr_radius_total(h)
            offsets = np.zeros(q.shape[0] + 1, dtype=np.int64)
            keys = np.zeros(total, dtype=np.uint64)
            self.R.qr_radius_copy(h, _ptr(offsets), _ptr(keys))
        finally:
            self.R.qr_radius_free(h)
        return offsets, keys, qms.value

    def scene(self, kind: str, items, closest_q, knn_q, kk: int, radius_q, r: float, rays=None,
              threads: int = 0):
        """Every query set of one scene on one reference structure (built once): returns
        {closest, knn, radius: (offsets, keys), rays (triangles)} and the times
        {build_ms, closest_ms, knn_ms, radius_ms, rays_ms}."""
        k = KIND[kind]
        items = _f32(items).reshape(-1, STRIDE[k])
        qc = _f32(closest_q).reshape(-1, 3)
        qk = _f32(knn_q).reshape(-1, 3)
        qr = _f32(radius_q).reshape(-1, 3)
        rays = np.zeros((0, 8), np.float32) if rays is None else _f32(rays).reshape(-1, 8)
        oc = np.zeros((qc.shape[0], 2), dtype=np.uint32)
        ok = np.zeros((qk.shape[0], kk, 2), dtype=np.uint32)
        orr = np.zeros(rays.shape[0], dtype=np.uint64)
        bms = ctypes.c_double(0.0)
        ms = (ctypes.c_double * 4)()
        h = self.R.qr_scene(k, _ptr(items), items.shape[0], _ptr(qc), qc.shape[0], _ptr(oc),
                            _ptr(qk), qk.shape[0], kk, _ptr(ok), _ptr(qr), qr.shape[0], r,
                            _ptr(rays), rays.shape[0], _ptr(orr), threads, ctypes.byref(bms), ms)
        try:
            total = self.R.qr_radius_total(h)
            offsets = np.zeros(qr.shape[0] + 1, dtype=np.int64)
            keys = np.zeros(total, dtype=np.uint64)
            self.R.qr_radius_copy(h, _ptr(offsets), _ptr(keys))
        finally:
            self.R.qr_radius_free(h)
        out = {"closest": oc, "knn": ok, "radius": (offsets, keys)}
        if k == 0:
            out["rays"] = orr
        times = {"build_ms": bms.value, "closest_ms": ms[0], "knn_ms": ms[1], "radius_ms": ms[2],
                 "rays_ms": ms[3]}
        return out, times

    def closest_brute(self, kind: str, items, q):
        k = KIND[kind]
        items = _f32(items).reshape(-1, STRIDE[k])
        q = _f32(q).reshape(-1, 3)
        out = np.zeros((q.shape[0], 2), dtype=np.uint32)
        self.R.qr_closest_brute(k, _ptr(items), items.shape[0], _ptr(q), q.shape[0], _ptr(out))
        return out

    def ray_hash(self, res):
        res = np.ascontiguousarray(res, dtype=np.uint64)
        hits = ctypes.c_uint64(0)
        return self.R.qr_ray_hash(_ptr(res), res.size, ctypes.byref(hits)), hits.value

    def closest_hash(self, res2):
        res2 = np.ascontiguousarray(res2, dtype=np.uint32).reshape(-1, 2)
        return self.R.qr_closest_hash(_ptr(res2), res2.shape[0])

    def list_hash(self, offsets, keys):
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        return self.R.qr_list_hash(_ptr(offsets), _ptr(keys), offsets.size - 1)

    def leaf(self):
        return self.R


def knn_to_csr(res: np.ndarray):
    """kNN rows (padded with id -1) -> (offsets, keys) in the radius CSR form."""
    ids = res[..., 1].view(np.int32)
    valid = ids >= 0
    counts = valid.sum(axis=1)
    offsets = np.zeros(res.shape[0] + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    keys = (res[..., 0].astype(np.uint64) << np.uint64(32)) | res[..., 1].astype(np.uint64)
    return offsets, keys[valid]


