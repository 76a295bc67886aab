"""ctypes binding of the engine's C ABI (include/quarry_b200.h) over torch device memory.

This is the foreign-function view of the engine: every call goes through an extern "C"
entry point of libquarry_b200.so with plain device pointers, sizes, a workspace and a CUDA
stream.  torch only provides device allocations and the current stream.

There is no fallback: when the shared library is missing or no CUDA device is present the
calls raise.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libquarry_b200.so"

QK_OK = 0
QK_TRI, QK_POINT, QK_GAUSS = 0, 1, 2
QK_BUILD_LBVH, QK_BUILD_SAH, QK_BUILD_SAH4 = 0, 1, 2
BUILDERS = {"lbvh": QK_BUILD_LBVH, "sah": QK_BUILD_SAH, "sah4": QK_BUILD_SAH4}
QK_ORDER_MORTON, QK_ORDER_DIRECTION, QK_WIDE, QK_ORDER_COHERENT = 1, 2, 4, 8
QK_TUNE_DYNAMIC, QK_TUNE_HIGH_OCC, QK_TUNE_SPLIT, QK_TUNE_SHORT_STACK = 256, 512, 1024, 2048
QK_TUNE_LEAF4 = 4096
QK_TUNE_STASH = 8192
QK_TUNE_TAIL = 16384
QK_TUNE_SPLIT8 = 32768
QK_TUNE_SPLIT4 = 65536
QK_SCHEDULE_BATCHED, QK_SCHEDULE_LOOP = 0, 1
QK_OP_RAY, QK_OP_CLOSEST, QK_OP_KNN, QK_OP_RADIUS = 0, 1, 2, 3
KINDS = {"tri": QK_TRI, "point": QK_POINT, "gauss": QK_GAUSS}
STRIDE = {QK_TRI: 9, QK_POINT: 3, QK_GAUSS: 10}

_P = ctypes.c_void_p
_I = ctypes.c_int
_U = ctypes.c_uint
_F = ctypes.c_float
_SZ = ctypes.c_size_t


class QkTree(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("n", ctypes.c_int32), ("depth", ctypes.c_int32),
                ("wide_count", ctypes.c_int32), ("nodes", _P), ("items", _P), ("prim_ids", _P),
                ("parent", _P), ("depth_arr", _P), ("bnodes", _P), ("leaves", _P),
                ("slot_of", _P), ("flags", _P), ("wide", _P), ("wide_id", _P),
                ("wide_leaf", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class QkTreeSizes(ctypes.Structure):
    _fields_ = [(name, _SZ) for name in ("nodes", "items", "prim_ids", "parent", "depth_arr",
                                          "bnodes", "leaves", "slot_of", "flags", "wide",
                                          "wide_id")]


class QkBatchTune(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("short_stack", ctypes.c_int32), ("chunks_per_fetch", ctypes.c_int32),
                ("split", ctypes.c_int32)]


class QkBatchIo(ctypes.Structure):
    _fields_ = [("input", _P), ("out", _P), ("offsets", _P), ("capacity", ctypes.c_int64),
                ("k", ctypes.c_int32), ("pad", ctypes.c_int32)]


class QkTopoEdit(ctypes.Structure):
    _fields_ = [("deleted", _P), ("n_deleted", ctypes.c_int32), ("inserted", _P),
                ("n_inserted", ctypes.c_int32), ("appended", ctypes.c_int32), ("moved", _P),
                ("n_moved", ctypes.c_int32), ("extra_items", _P), ("moved_items", _P)]


class QkTopoInfo(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int32) for name in ("rebuild", "cuts", "old_leaves",
                                                    "new_leaves", "max_cut", "spliced", "depth",
                                                    "reason")]


_PP = ctypes.POINTER(ctypes.c_void_p)
_I64P = ctypes.POINTER(ctypes.c_int64)

EXPORTS = {
    "qk_status_string": (ctypes.c_char_p, [_I]),
    "qk_last_error": (ctypes.c_char_p, []),
    "qk_describe": (_I, [ctypes.c_char_p, _I]),
    "qk_stride_floats": (_I, [_I]),
    "qk_leaf_vec4": (_I, [_I]),
    "qk_tree_bytes": (_I, [_I, _I, ctypes.POINTER(QkTreeSizes)]),
    "qk_build_workspace_bytes": (_SZ, [_I, _I, _I]),
    "qk_query_workspace_bytes": (_SZ, [_I, _U]),
    "qk_radius_workspace_bytes": (_SZ, [_I, _U]),
    "qk_build": (_I, [ctypes.POINTER(QkTree), _I, _I, _P, _P, _SZ, _P]),
    "qk_refit": (_I, [ctypes.POINTER(QkTree), _P, _P, _SZ, _P]),
    "qk_refit_dirty": (_I, [ctypes.POINTER(QkTree), _P, _P, _I, _P, _SZ, _P]),
    "qk_wide_build": (_I, [ctypes.POINTER(QkTree), _P, _SZ, _P]),
    "qk_wide_build_leaf4": (_I, [ctypes.POINTER(QkTree), _P, _SZ, _P]),
    "qk_update_workspace_bytes": (_SZ, [_I, _I, _I, _I]),
    "qk_update_topology": (_I, [ctypes.POINTER(QkTree), ctypes.POINTER(QkTree),
                                ctypes.POINTER(QkTopoEdit), _I, _I, ctypes.POINTER(QkTopoInfo),
                                _P, _SZ, _P]),
    "qk_raycast": (_I, [ctypes.POINTER(QkTree), _P, _I, _P, _U, _P, _P, _SZ, _P]),
    "qk_closest": (_I, [ctypes.POINTER(QkTree), _P, _I, _P, _U, _P, _P, _SZ, _P]),
    "qk_knn": (_I, [ctypes.POINTER(QkTree), _P, _I, _I, _I, _P, _U, _P, _P, _SZ, _P]),
    "qk_radius_count": (_I, [ctypes.POINTER(QkTree), _P, _I, _F, _P,
                             ctypes.POINTER(ctypes.c_int64), _U, _P, _P, _SZ, _P]),
    "qk_radius_fill": (_I, [ctypes.POINTER(QkTree), _P, _I, _F, _P, _P, _U, _P, _SZ, _P]),
    "qk_validate": (_I, [ctypes.POINTER(QkTree), _P, _P, _P, _SZ, _P]),
    "qk_validate_workspace_bytes": (_SZ, [_I]),
    "qk_sort_workspace_bytes": (_SZ, [_I]),
    "qk_raycast_ids": (_I, [ctypes.POINTER(QkTree), _P, _I, _P, _P, _U, _P, _SZ, _P]),
    "qk_grad_workspace_bytes": (_SZ, [_I, _I]),
    "qk_distance_grad": (_I, [ctypes.POINTER(QkTree), _P, _P, _P, _P, _I, _P, _P, _P, _SZ, _P]),
    "qk_ray_t_grad": (_I, [ctypes.POINTER(QkTree), _P, _P, _P, _P, _I, _P, _P, _P, _SZ, _P]),
    "qk_segment_sum": (_I, [_P, _P, _I, _I, _I, _P, _P, _SZ, _P]),
    "qk_grad_vertices_workspace_bytes": (_SZ, [_I]),
    "qk_ray_t_grad_vertices": (_I, [ctypes.POINTER(QkTree), _P, _P, _P, _P, _I, _P, _I, _P, _P,
                                    _P, _SZ, _P]),
    "qk_distance_grad_vertices": (_I, [ctypes.POINTER(QkTree), _P, _P, _P, _P, _I, _P, _I, _P,
                                       _P, _P, _SZ, _P]),
    "qk_raycast_noalloc": (_I, [ctypes.POINTER(QkTree), _P, _I, _P, _U, _P]),
    "qk_raycast_mapped": (_I, [ctypes.POINTER(QkTree), _P, _I, _P, _U, _P, _SZ, _P]),
    "qk_raycast_host_workspace_bytes": (_SZ, [_I, _I]),
    "qk_raycast_host": (_I, [ctypes.POINTER(QkTree), _P, _I, _P, _P, _P, _I, _U, _P, _SZ, _P, _P,
                             _P, _P]),
    "qk_sort_pairs": (_I, [_P, _P, _P, _P, _I, _I, _P, _SZ, _P]),
    "qk_batch_arena_bytes": (_SZ, [_I, _P, _I, _U]),
    "qk_batch_create": (_I, [_PP, _I, _P, _I, _P, _P, _SZ, _U, _P]),
    "qk_batch_build": (_I, [_P, _U, _P]),
    "qk_batch_build_sah": (_I, [_P, _I, _P]),
    "qk_batch_sync": (_I, [_P, _P]),
    "qk_batch_tree": (_I, [_P, _I, ctypes.POINTER(QkTree)]),
    "qk_batch_scenes": (_I, [_P]),
    "qk_batch_destroy": (None, [_P]),
    "qk_batch_plan_bytes": (_SZ, [_P, _I, _P, _U]),
    "qk_batch_plan_create": (_I, [_PP, _P, _I, _P, _P, _P, _SZ, _U, _P]),
    "qk_batch_query": (_I, [_P, ctypes.POINTER(QkBatchIo), ctypes.POINTER(QkBatchTune), _U, _P]),
    "qk_batch_plan_status": (_I, [_P, _I64P, _I64P, _P]),
    "qk_batch_plan_destroy": (None, [_P]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libquarry_b200.so and declare every export of include/quarry_b200.h."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is not built; run quarry-gpu_b200/build.py")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in EXPORTS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class QkError(RuntimeError):
    def __init__(self, status: int, where: str):
        L = lib()
        msg = L.qk_last_error().decode(errors="replace")
        super().__init__(f"{where}: {L.qk_status_string(status).decode()} ({msg})")
        self.status = status


def check(status: int, where: str) -> None:
    if status != QK_OK:
        raise QkError(status, where)


def describe() -> str:
    buf = ctypes.create_string_buffer(256)
    return buf.value.decode() if lib().qk_describe(buf, 256) else ""


# ---------------------------------------------------------------------------------------
# torch-backed device objects
# ---------------------------------------------------------------------------------------
def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the B200 engine needs a CUDA device")
    return torch


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _stream():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev_bytes(nbytes: int):
    torch = _torch()
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")


def to_device(a: np.ndarray, dtype=None):
    torch = _torch()
    a = np.ascontiguousarray(a if dtype is None else a.astype(dtype, copy=False))
    return torch.from_numpy(a).to("cuda")


class Workspace:
    """A growable device scratch buffer reused across calls."""

    def __init__(self):
        self.buf = None

    def get(self, nbytes: int):
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = _dev_bytes(max(nbytes, 1 << 16))
        return self.buf


class DeviceTree:
    """One tree: device arrays allocated from torch, filled by qk_build.

    kind: "tri" | "point" | "gauss"; items: (n, stride) float32 in scene order (numpy or a
    CUDA tensor).  builder: "lbvh", "sah" or "sah4" (leaf-size-4 SAH)."""

    def __init__(self, kind: str, items, builder: str = "lbvh", sah_bins: int = 32):
        torch = _torch()
        L = lib()
        self.kind = KINDS[kind]
        if isinstance(items, np.ndarray):
            items = to_device(items.reshape(-1, STRIDE[self.kind]), np.float32)
        self.items_scene = items.reshape(-1, STRIDE[self.kind]).contiguous()
        n = self.items_scene.shape[0]
        self.n = n
        self.arrays, self.t = self._alloc(n)
        self.ws = Workspace()
        if builder not in BUILDERS:
            raise ValueError(f"builder must be one of {sorted(BUILDERS)}")
        self.builder = BUILDERS[builder]
        self.sah_bins = sah_bins
        self.build()
        del torch, L

    def _alloc(self, n: int):
        sizes = QkTreeSizes()
        check(lib().qk_tree_bytes(self.kind, n, ctypes.byref(sizes)), "qk_tree_bytes")
        arrays = {}
        for name in ("nodes", "items", "prim_ids", "parent", "depth_arr", "bnodes", "leaves",
                     "slot_of", "flags", "wide_id"):
            arrays[name] = _dev_bytes(getattr(sizes, name))
        arrays["flags"].zero_()
        t = QkTree()
        t.kind = self.kind
        t.n = n
        for name, buf in arrays.items():
            setattr(t, name, buf.data_ptr())
        t.wide = None
        return arrays, t

    # ---- build / refit ----
    def _build_ws(self):
        nb = lib().qk_build_workspace_bytes(self.kind, self.n, self.builder)
        return self.ws.get(nb), nb

    def build(self) -> None:
        ws, nb = self._build_ws()
        check(lib().qk_build(ctypes.byref(self.t), self.builder, self.sah_bins,
                             _ptr(self.items_scene), _ptr(ws), ws.numel(), _stream()), "qk_build")

    @property
    def depth(self) -> int:
        return self.t.depth

    def build_wide(self, leaf4: bool = False) -> int:
        """4-wide nodes (qk_wide_build), or with leaf4 the leaf-size-4 form
        (qk_wide_build_leaf4: subtrees of 2..4 primitives on contiguous slots are one leaf
        slot).  Returns the node count."""
        ws, _ = self._build_ws()
        fn = lib().qk_wide_build_leaf4 if leaf4 else lib().qk_wide_build
        name = "qk_wide_build_leaf4" if leaf4 else "qk_wide_build"
        self.t.wide = None
        check(fn(ctypes.byref(self.t), _ptr(ws), ws.numel(), _stream()), name + " (count)")
        self.arrays["wide"] = _dev_bytes(self.t.wide_count * 128)
        self.t.wide = self.arrays["wide"].data_ptr()
        check(fn(ctypes.byref(self.t), _ptr(ws), ws.numel(), _stream()), name)
        return self.t.wide_count

    def refit(self, items) -> None:
        if isinstance(items, np.ndarray):
            items = to_device(items.reshape(-1, STRIDE[self.kind]), np.float32)
        self.items_scene = items.reshape(-1, STRIDE[self.kind]).contiguous()
        ws, _ = self._build_ws()
        check(lib().qk_refit(ctypes.byref(self.t), _ptr(self.items_scene), _ptr(ws), ws.numel(),
                             _stream()), "qk_refit")

    def refit_dirty(self, ids, items_subset) -> None:
        if isinstance(ids, np.ndarray):
            ids = to_device(ids, np.int32)
        if isinstance(items_subset, np.ndarray):
            items_subset = to_device(items_subset.reshape(-1, STRIDE[self.kind]), np.float32)
        ws, _ = self._build_ws()
        check(lib().qk_refit_dirty(ctypes.byref(self.t), _ptr(ids), _ptr(items_subset),
                                   int(ids.numel()), _ptr(ws), ws.numel(), _stream()),
              "qk_refit_dirty")

    def update_topology(self, new_items, deleted=(), inserted=(), moved=(), cut_size: int = 0):
        """Topology edit (qk_update_topology) toward the new scene `new_items` (scene order):
        deleted old indices, inserted new indices, moved new indices; the appended count
        follows from the sizes.  Surgery when the plan accepts, else a full rebuild.  Returns
        the plan's qk_topo_info fields as a dict.  The wide layer is dropped."""
        torch = _torch()
        if isinstance(new_items, np.ndarray):
            new_items = to_device(new_items.reshape(-1, STRIDE[self.kind]), np.float32)
        new_items = new_items.reshape(-1, STRIDE[self.kind]).contiguous()
        n_new = new_items.shape[0]
        dele = torch.as_tensor(np.asarray(deleted, np.int32).reshape(-1), device="cuda")
        ins = torch.as_tensor(np.asarray(inserted, np.int32).reshape(-1), device="cuda")
        mov = torch.as_tensor(np.asarray(moved, np.int32).reshape(-1), device="cuda")
        appended = n_new - self.n + dele.numel() - ins.numel()
        extra_idx = torch.cat([ins.long(), torch.arange(n_new - appended, n_new, device="cuda")])
        extra = new_items[extra_idx].contiguous()
        moved_items = new_items[mov.long()].contiguous()
        e = QkTopoEdit(_ptr(dele), dele.numel(), _ptr(ins), ins.numel(), int(appended), _ptr(mov),
                       mov.numel(), _ptr(extra), _ptr(moved_items))
        arrays, t = self._alloc(n_new)
        nb = lib().qk_update_workspace_bytes(self.kind, self.n, n_new, int(extra.shape[0]))
        ws = _dev_bytes(nb)
        info = QkTopoInfo()
        check(lib().qk_update_topology(ctypes.byref(self.t), ctypes.byref(t), ctypes.byref(e),
                                       int(cut_size), self.sah_bins, ctypes.byref(info), _ptr(ws),
                                       ws.numel(), _stream()), "qk_update_topology")
        out = {name: getattr(info, name) for name, _ in QkTopoInfo._fields_}
        self.arrays, self.t, self.n, self.items_scene = arrays, t, n_new, new_items
        if info.rebuild:
            self.build()
        return out

    # ---- read-back ----
    def host(self, name: str, dtype, count: int | None = None) -> np.ndarray:
        buf = self.arrays[name]
        a = buf.cpu().numpy().view(dtype)
        return a if count is None else a[:count]

    def nodes_bytes(self) -> np.ndarray:
        return self.arrays["nodes"].cpu().numpy()[: (2 * self.n - 1) * 32]

    def validate(self) -> list[int]:
        torch = _torch()
        err = torch.zeros(8, dtype=torch.int32, device="cuda")
        nb = lib().qk_validate_workspace_bytes(self.n)
        ws = _dev_bytes(nb)
        check(lib().qk_validate(ctypes.byref(self.t), _ptr(self.items_scene), _ptr(err), _ptr(ws),
                                ws.numel(), _stream()), "qk_validate")
        return err.cpu().tolist()

    # ---- queries (device in, device out) ----
    def raycast(self, rays, flags: int = 0, stats=None, out=None, ws=None):
        torch = _torch()
        count = rays.shape[0]
        if out is None:
            out = torch.empty(count, dtype=torch.int64, device="cuda")
        nb = lib().qk_query_workspace_bytes(count, flags)
        w = ws if ws is not None else self.ws.get(nb)
        check(lib().qk_raycast(ctypes.byref(self.t), _ptr(rays), count, _ptr(out), flags,
                               _ptr(stats), _ptr(w), w.numel(), _stream()), "qk_raycast")
        return out

    def raycast_mapped(self, host_rays, host_out, flags: int = 0, ws=None):
        """Zero-copy ray query: the traversal reads pinned host rays and writes pinned host
        results directly; synchronise the current stream before reading host_out."""
        count = host_rays.shape[0]
        w = ws if ws is not None else self.ws.get(lib().qk_query_workspace_bytes(count, flags))
        check(lib().qk_raycast_mapped(ctypes.byref(self.t), _ptr(host_rays), count,
                                      _ptr(host_out), flags, _ptr(w), w.numel(), _stream()),
              "qk_raycast_mapped")
        return host_out

    def raycast_host(self, host_rays, host_out, dev_rays, dev_out, flags: int = 0,
                     chunks: int = 8, streams=None, ws=None):
        """Pipelined host -> device -> host ray query (pinned buffers): uploads on
        streams[0], traversals alternating between streams[1] and [2], read-backs on
        streams[3]; synchronise streams[3] before reading host_out."""
        torch = _torch()
        count = host_rays.shape[0]
        if streams is None:
            streams = tuple(torch.cuda.Stream() for _ in range(4))
        if ws is None:
            ws = self.ws.get(lib().qk_raycast_host_workspace_bytes(count, chunks))
        check(lib().qk_raycast_host(ctypes.byref(self.t), _ptr(host_rays), count, _ptr(host_out),
                                    _ptr(dev_rays), _ptr(dev_out), chunks, flags, _ptr(ws),
                                    ws.numel(), *(ctypes.c_void_p(x.cuda_stream) for x in streams)),
              "qk_raycast_host")
        return streams

    def raycast_ids(self, rays, flags: int = 0):
        """First hits with the hit primitive (scene index, -1 on a miss)."""
        torch = _torch()
        count = rays.shape[0]
        out = torch.empty(count, dtype=torch.int64, device="cuda")
        ids = torch.empty(count, dtype=torch.int32, device="cuda")
        w = self.ws.get(lib().qk_query_workspace_bytes(count, flags))
        check(lib().qk_raycast_ids(ctypes.byref(self.t), _ptr(rays), count, _ptr(out), _ptr(ids),
                                   flags, _ptr(w), w.numel(), _stream()), "qk_raycast_ids")
        return out, ids

    def distance_grad(self, pts, results, grad_dist=None):
        """Adjoint of the distances of qk_closest's results: (grad_points, grad_items)."""
        torch = _torch()
        count = pts.shape[0]
        gp = torch.empty((count, 3), dtype=torch.float32, device="cuda")
        gi = torch.empty_like(self.items_scene)
        w = _dev_bytes(lib().qk_grad_workspace_bytes(count, STRIDE[self.kind]))
        check(lib().qk_distance_grad(ctypes.byref(self.t), _ptr(self.items_scene), _ptr(pts),
                                     _ptr(results), _ptr(grad_dist), count, _ptr(gp), _ptr(gi),
                                     _ptr(w), w.numel(), _stream()), "qk_distance_grad")
        return gp, gi

    def ray_t_grad(self, rays, ids, grad_t=None, with_rays: bool = True):
        """Adjoint of the first-hit t: (grad_tris (n, 9), grad_rays (count, 6) or None)."""
        torch = _torch()
        count = rays.shape[0]
        gt = torch.empty((self.n, 9), dtype=torch.float32, device="cuda")
        gr = torch.empty((count, 6), dtype=torch.float32, device="cuda") if with_rays else None
        w = _dev_bytes(lib().qk_grad_workspace_bytes(count, 9))
        check(lib().qk_ray_t_grad(ctypes.byref(self.t), _ptr(self.items_scene), _ptr(rays),
                                  _ptr(ids), _ptr(grad_t), count, _ptr(gt), _ptr(gr), _ptr(w),
                                  w.numel(), _stream()), "qk_ray_t_grad")
        return gt, gr

    def ray_t_grad_vertices(self, rays, ids, indices, nverts: int, grad_t=None,
                            with_rays: bool = True):
        """Adjoint of the first-hit t summed per mesh vertex in FP64: (grad_verts (nverts, 3),
        grad_rays (count, 6) or None); indices (n, 3) int32 corner vertex ids."""
        torch = _torch()
        count = rays.shape[0]
        gv = torch.empty((nverts, 3), dtype=torch.float32, device="cuda")
        gr = torch.empty((count, 6), dtype=torch.float32, device="cuda") if with_rays else None
        idx = indices.to(torch.int32).contiguous()
        w = _dev_bytes(lib().qk_grad_vertices_workspace_bytes(count))
        check(lib().qk_ray_t_grad_vertices(ctypes.byref(self.t), _ptr(self.items_scene), _ptr(rays),
                                           _ptr(ids), _ptr(grad_t), count, _ptr(idx), nverts,
                                           _ptr(gv), _ptr(gr), _ptr(w), w.numel(), _stream()),
              "qk_ray_t_grad_vertices")
        return gv, gr

    def distance_grad_vertices(self, pts, results, indices, nverts: int, grad_dist=None):
        """Adjoint of the triangle distances summed per mesh vertex in FP64:
        (grad_points (count, 3), grad_verts (nverts, 3))."""
        torch = _torch()
        count = pts.shape[0]
        gp = torch.empty((count, 3), dtype=torch.float32, device="cuda")
        gv = torch.empty((nverts, 3), dtype=torch.float32, device="cuda")
        idx = indices.to(torch.int32).contiguous()
        w = _dev_bytes(lib().qk_grad_vertices_workspace_bytes(count))
        check(lib().qk_distance_grad_vertices(ctypes.byref(self.t), _ptr(self.items_scene),
                                              _ptr(pts), _ptr(results), _ptr(grad_dist), count,
                                              _ptr(idx), nverts, _ptr(gp), _ptr(gv), _ptr(w),
                                              w.numel(), _stream()), "qk_distance_grad_vertices")
        return gp, gv

    def closest(self, pts, flags: int = 0, stats=None, out=None):
        torch = _torch()
        count = pts.shape[0]
        if out is None:
            out = torch.empty((count, 2), dtype=torch.int32, device="cuda")
        nb = lib().qk_query_workspace_bytes(count, flags)
        w = self.ws.get(nb)
        check(lib().qk_closest(ctypes.byref(self.t), _ptr(pts), count, _ptr(out), flags,
                               _ptr(stats), _ptr(w), w.numel(), _stream()), "qk_closest")
        return out

    def knn(self, pts, k: int, flags: int = 0, stats=None, out=None, stride: int | None = None):
        torch = _torch()
        count = pts.shape[0]
        stride = k if stride is None else stride
        if out is None:
            out = torch.empty((count, stride, 2), dtype=torch.int32, device="cuda")
        nb = lib().qk_query_workspace_bytes(count, flags)
        w = self.ws.get(nb)
        check(lib().qk_knn(ctypes.byref(self.t), _ptr(pts), count, k, stride, _ptr(out), flags,
                           _ptr(stats), _ptr(w), w.numel(), _stream()), "qk_knn")
        return out

    def radius(self, pts, r: float, flags: int = 0, stats=None):
        torch = _torch()
        count = pts.shape[0]
        offsets = torch.empty(count + 1, dtype=torch.int32, device="cuda")
        nb = lib().qk_radius_workspace_bytes(count, flags)
        w = self.ws.get(nb)
        total = ctypes.c_int64(0)
        check(lib().qk_radius_count(ctypes.byref(self.t), _ptr(pts), count, float(r),
                                    _ptr(offsets), ctypes.byref(total), flags, _ptr(stats),
                                    _ptr(w), w.numel(), _stream()), "qk_radius_count")
        keys = torch.empty(max(total.value, 1), dtype=torch.int64, device="cuda")
        check(lib().qk_radius_fill(ctypes.byref(self.t), _ptr(pts), count, float(r),
                                   _ptr(offsets), _ptr(keys), flags, _ptr(w), w.numel(),
                                   _stream()), "qk_radius_fill")
        return offsets, keys[: total.value]


def segment_sum(keys, values, segments: int):
    """Deterministic out[k] = sum of values[i] with keys[i] == k, in increasing i."""
    torch = _torch()
    count = keys.numel()
    ch = values.shape[1] if values.dim() > 1 else 1
    out = torch.empty((segments, ch), dtype=torch.float32, device="cuda")
    w = _dev_bytes(lib().qk_grad_workspace_bytes(count, 0))
    check(lib().qk_segment_sum(_ptr(keys), _ptr(values), count, ch, segments, _ptr(out), _ptr(w),
                               w.numel(), _stream()), "qk_segment_sum")
    return out


def sort_pairs(keys, vals, bits: int = 32):
    """Stable radix sort of uint32 (key, value) tensors on the device (returns copies)."""
    torch = _torch()
    n = keys.numel()
    kin, vin = keys.clone(), vals.clone()
    kout, vout = torch.empty_like(kin), torch.empty_like(vin)
    nb = lib().qk_sort_workspace_bytes(n)
    ws = _dev_bytes(nb)
    check(lib().qk_sort_pairs(_ptr(kin), _ptr(vin), _ptr(kout), _ptr(vout), n, bits, _ptr(ws),
                              ws.numel(), _stream()), "qk_sort_pairs")
    return kout, vout


# ---------------------------------------------------------------------------------------
# batched scenes
# ---------------------------------------------------------------------------------------
class Batch:
    """Scenes of one primitive kind built and queried together (qk_batch_*).

    scenes: list of (n_s, stride) float32 arrays (numpy or CUDA tensors).  wide=True also
    builds every scene's 4-wide nodes."""

    def __init__(self, kind: str, scenes, wide: bool = False):
        torch = _torch()
        self.kind = KINDS[kind]
        st = STRIDE[self.kind]
        parts = [np.asarray(a, np.float32).reshape(-1, st) if isinstance(a, np.ndarray)
                 else a.reshape(-1, st) for a in scenes]
        self.counts = np.array([p.shape[0] for p in parts], dtype=np.int32)
        if isinstance(parts[0], np.ndarray):
            self.items = to_device(np.concatenate(parts, axis=0), np.float32)
        else:
            self.items = torch.cat(parts, dim=0).contiguous()
        self.scenes = len(parts)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.flags = QK_WIDE if wide else 0
        L = lib()
        nb = L.qk_batch_arena_bytes(self.kind, self.counts.ctypes.data, self.scenes, self.flags)
        if nb == 0:
            raise QkError(1, "qk_batch_arena_bytes")
        self.arena = _dev_bytes(nb)
        self.h = ctypes.c_void_p()
        check(L.qk_batch_create(ctypes.byref(self.h), self.kind, self.counts.ctypes.data,
                                self.scenes, _ptr(self.items), _ptr(self.arena), nb, self.flags,
                                _stream()), "qk_batch_create")

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value and _lib is not None:
            _lib.qk_batch_destroy(h)
            self.h = None

    def build(self, schedule: int = QK_SCHEDULE_BATCHED) -> None:
        check(lib().qk_batch_build(self.h, schedule, _stream()), "qk_batch_build")

    def build_sah(self, bins: int = 32) -> None:
        """Every scene with the binned SAH builder, scene by scene (synchronizes)."""
        check(lib().qk_batch_build_sah(self.h, bins, _stream()), "qk_batch_build_sah")

    def sync(self) -> None:
        check(lib().qk_batch_sync(self.h, _stream()), "qk_batch_sync")

    def tree(self, s: int) -> QkTree:
        t = QkTree()
        check(lib().qk_batch_tree(self.h, s, ctypes.byref(t)), "qk_batch_tree")
        return t

    def view(self, s: int) -> "DeviceTree":
        """Scene s as a DeviceTree (no copy): single-tree queries, validation, read-back."""
        t = self.tree(s)
        v = DeviceTree.__new__(DeviceTree)
        v.kind = self.kind
        v.n = t.n
        v.t = t
        v.items_scene = self.items[int(self.offsets[s]):int(self.offsets[s + 1])]
        sizes = QkTreeSizes()
        check(lib().qk_tree_bytes(self.kind, t.n, ctypes.byref(sizes)), "qk_tree_bytes")
        base = self.arena.data_ptr()
        v.arrays = {}
        for name in ("nodes", "items", "prim_ids", "parent", "depth_arr", "bnodes", "leaves",
                     "slot_of", "flags", "wide", "wide_id"):
            ptr = getattr(t, name)
            if ptr:
                off = ptr - base
                v.arrays[name] = self.arena[off:off + getattr(sizes, name)]
        v.ws = Workspace()
        v.builder = QK_BUILD_LBVH
        v.sah_bins = 32
        v.owner = self
        return v

    def plan(self, op: int, counts, params=None, flags: int = 0) -> "BatchPlan":
        return BatchPlan(self, op, counts, params, flags)


class BatchPlan:
    """Per-scene query counts of one operation over a Batch (qk_batch_plan_*)."""

    def __init__(self, batch: Batch, op: int, counts, params=None, flags: int = 0):
        L = lib()
        self.batch = batch
        self.op = op
        self.counts = np.ascontiguousarray(counts, dtype=np.int32)
        self.total = int(self.counts.sum())
        self.q_off = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.params = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        nb = L.qk_batch_plan_bytes(batch.h, op, self.counts.ctypes.data, flags)
        self.mem = _dev_bytes(nb)
        self.h = ctypes.c_void_p()
        check(L.qk_batch_plan_create(ctypes.byref(self.h), batch.h, op, self.counts.ctypes.data,
                                     None if self.params is None else self.params.ctypes.data,
                                     _ptr(self.mem), nb, flags, _stream()), "qk_batch_plan_create")

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value and _lib is not None:
            _lib.qk_batch_plan_destroy(h)
            self.h = None

    def query(self, inputs, out, offsets=None, capacity: int = 0, k: int = 0, tune=None,
              schedule: int = QK_SCHEDULE_BATCHED) -> None:
        io = QkBatchIo()
        io.input = _ptr(inputs)
        io.out = _ptr(out)
        io.offsets = _ptr(offsets)
        io.capacity = int(capacity)
        io.k = int(k)
        tp = None
        if tune is not None:
            t = QkBatchTune()
            t.block, t.blocks_per_sm, t.short_stack, t.chunks_per_fetch = (
                int(tune["block"]), int(tune["blocks_per_sm"]), int(tune["short_stack"]),
                int(tune["chunks_per_fetch"]))
            t.split = int(tune.get("split", 0))
            tp = ctypes.byref(t)
        check(lib().qk_batch_query(self.h, ctypes.byref(io), tp, schedule, _stream()),
              "qk_batch_query")

    def status(self, raise_on_overrun: bool = True) -> tuple[int, int]:
        """(radius keys of the last query or -1, traversals stopped by a limit); raises on a
        radius capacity overrun unless raise_on_overrun is False."""
        tot = ctypes.c_int64(0)
        ovf = ctypes.c_int64(0)
        st = lib().qk_batch_plan_status(self.h, ctypes.byref(tot), ctypes.byref(ovf), _stream())
        if st != QK_OK and (raise_on_overrun or st != 3):
            check(st, "qk_batch_plan_status")
        return tot.value, ovf.value
