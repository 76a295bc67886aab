"""Zero-copy CUDA path of the module's classes (Scene, PointCloud, GaussianCloud).

The reference module takes host arrays, so every query pays an upload, a download and a
synchronisation.  Here the same methods also accept device arrays -- torch CUDA tensors,
objects with `__cuda_array_interface__` (CuPy, Numba) or CUDA DLPack capsules -- and then
run entirely on the device: inputs are read in place, results come back as torch CUDA
tensors, and the work is enqueued on torch's current stream without a host synchronisation
(except radius, whose result size is read back, as the C ABI's count / fill split requires).
Host inputs keep the original behaviour.  The queries go through the C ABI
(include/quarry_b200.h) on the object's own tree; results are the same bits as the host path.
`last_query_ms` is not updated by device calls (nothing is timed or synchronised).
"""
from __future__ import annotations

import ctypes
import math

from . import capi

_ORDERS = {"input": 0, "morton": capi.QK_ORDER_MORTON}
_RAY_ORDERS = {"input": 0, "morton": capi.QK_ORDER_MORTON,
               "direction": capi.QK_ORDER_DIRECTION}
_FIELDS = ("nodes", "items", "prim_ids", "parent", "depth_arr", "bnodes", "leaves", "slot_of",
           "flags", "wide", "wide_id")


def as_cuda(x):
    """A torch CUDA tensor viewing `x` without a copy, or None when `x` lives on the host."""
    try:
        import torch
    except ImportError:
        return None
    if isinstance(x, torch.Tensor):
        return x if x.is_cuda else None
    if hasattr(x, "__cuda_array_interface__"):
        return torch.as_tensor(x, device="cuda")
    if hasattr(x, "__dlpack__") and hasattr(x, "__dlpack_device__"):
        if int(x.__dlpack_device__()[0]) == 2:  # kDLCUDA
            return torch.from_dlpack(x)
    return None


def _points(x, name: str):
    import torch

    t = as_cuda(x)
    if t is None or t.dim() != 2 or t.shape[1] != 3:
        raise ValueError(f"{name} must be a CUDA array of shape (N, 3)")
    return t.to(torch.float32).contiguous()


def _tree(obj, wide: bool) -> capi.QkTree:
    v = obj._tree_view(wide)
    t = capi.QkTree()
    t.kind, t.n, t.depth, t.wide_count = v[0], v[1], v[2], v[3]
    for name, ptr in zip(_FIELDS, v[4:]):
        setattr(t, name, ptr or None)
    return t


def _flags(order: str, wide: bool, table=_ORDERS) -> int:
    if order not in table:
        raise ValueError(f"order must be one of {sorted(table)}")
    return table[order] | (capi.QK_WIDE if wide else 0)


def _ws(nbytes: int):
    import torch

    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")


def raycast(self, origins, dirs, tmax=math.inf, order="input", wide=False):
    import torch

    o = _points(origins, "origins")
    d = _points(dirs, "dirs")
    if o.shape[0] != d.shape[0]:
        raise ValueError("origins and dirs must match")
    n = o.shape[0]
    rays = torch.empty((n, 8), dtype=torch.float32, device=o.device)
    rays[:, 0:3] = o
    rays[:, 3:6] = d
    rays[:, 6] = 1e-6
    rays[:, 7] = tmax
    flags = _flags(order, wide, _RAY_ORDERS)
    t = _tree(self, wide)
    out = torch.empty(n, dtype=torch.int64, device=o.device)
    w = _ws(capi.lib().qk_query_workspace_bytes(n, flags))
    capi.check(capi.lib().qk_raycast(ctypes.byref(t), rays.data_ptr(), n, out.data_ptr(), flags,
                                     None, w.data_ptr(), w.numel(), capi._stream()), "raycast")
    hit = (out >> 32) != 0
    tt = (out & 0xFFFFFFFF).to(torch.int32).view(torch.float32)
    return hit, torch.where(hit, tt, torch.full_like(tt, math.inf))


def closest(self, points, order="input", wide=False):
    import torch

    p = _points(points, "points")
    n = p.shape[0]
    flags = _flags(order, wide)
    t = _tree(self, wide)
    out = torch.empty((n, 2), dtype=torch.int32, device=p.device)
    w = _ws(capi.lib().qk_query_workspace_bytes(n, flags))
    capi.check(capi.lib().qk_closest(ctypes.byref(t), p.data_ptr(), n, out.data_ptr(), flags, None,
                                     w.data_ptr(), w.numel(), capi._stream()), "closest")
    return out[:, 0].view(torch.float32), out[:, 1]


def knn(self, points, k, order="input", wide=False):
    import torch

    if not 1 <= int(k) <= 32:
        raise ValueError("k must be in [1, 32]")
    p = _points(points, "points")
    n = p.shape[0]
    flags = _flags(order, wide)
    t = _tree(self, wide)
    out = torch.empty((n, k, 2), dtype=torch.int32, device=p.device)
    w = _ws(capi.lib().qk_query_workspace_bytes(n, flags))
    capi.check(capi.lib().qk_knn(ctypes.byref(t), p.data_ptr(), n, k, k, out.data_ptr(), flags,
                                 None, w.data_ptr(), w.numel(), capi._stream()), "knn")
    return out[..., 0].view(torch.float32), out[..., 1]


def radius(self, points, radius, order="input", wide=False):
    import torch

    if not radius >= 0:
        raise ValueError("radius must be >= 0")
    p = _points(points, "points")
    n = p.shape[0]
    flags = _flags(order, wide)
    t = _tree(self, wide)
    offsets = torch.empty(n + 1, dtype=torch.int32, device=p.device)
    w = _ws(capi.lib().qk_radius_workspace_bytes(n, flags))
    total = ctypes.c_int64(0)
    capi.check(capi.lib().qk_radius_count(ctypes.byref(t), p.data_ptr(), n, float(radius),
                                          offsets.data_ptr(), ctypes.byref(total), flags, None,
                                          w.data_ptr(), w.numel(), capi._stream()), "radius count")
    keys = torch.empty(max(total.value, 1), dtype=torch.int64, device=p.device)
    capi.check(capi.lib().qk_radius_fill(ctypes.byref(t), p.data_ptr(), n, float(radius),
                                         offsets.data_ptr(), keys.data_ptr(), flags, w.data_ptr(),
                                         w.numel(), capi._stream()), "radius fill")
    keys = keys[: total.value]
    d2 = (keys >> 32).to(torch.int32).view(torch.float32)
    ids = (keys & 0xFFFFFFFF).to(torch.int32)
    return offsets.to(torch.int64), d2, ids


def install(*classes) -> None:
    """Give every class's query methods the device path (host inputs keep the original)."""
    for cls in classes:
        for name, dev, first_arg in (("raycast", raycast, "origins"), ("closest", closest, "points"),
                                     ("knn", knn, "points"), ("radius", radius, "points")):
            host = getattr(cls, name, None)
            if host is None or getattr(host, "_zero_copy", False):
                continue

            def method(self, *args, _host=host, _dev=dev, _first=first_arg, **kw):
                first = args[0] if args else kw.get(_first)
                if first is not None and as_cuda(first) is not None:
                    return _dev(self, *args, **kw)
                return _host(self, *args, **kw)

            method.__name__ = name
            method.__doc__ = (host.__doc__ or "") + (
                "\n\nDevice arrays (torch CUDA tensors, __cuda_array_interface__, CUDA DLPack) "
                "run without copies on torch's current stream and return torch CUDA tensors.")
            method._zero_copy = True
            setattr(cls, name, method)
