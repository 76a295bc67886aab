"""Differentiable spatial queries for PyTorch (CUDA tensors).

    d = quarry.torch.gaussian_distance(points, means, rotations, scales)
    d = quarry.torch.triangle_distance(points, vertices, indices)
    t, hit = quarry.torch.ray_hit_t(origins, dirs, vertices, indices)

Forward: the engine's bit-exact queries (closest primitive / first hit) over a tree built
from the current parameters.  Backward: the engine's adjoint kernels, which recompute only
the selected leaf test in FP64 and differentiate it (envelope theorem for distances, the
plane-crossing derivative for t); per-primitive and per-vertex sums are deterministic
(sorted, no float atomics) and stay in FP64 until one final rounding to FP32 (mesh vertices
are summed straight from the per-query terms, not through per-triangle FP32 sums).  Distances are Euclidean (not squared); d = 0 inside a solid
ellipsoid or on a triangle has gradient 0.  Rays that miss return t = inf and no gradient.
"""
from __future__ import annotations

import math

import torch

from . import capi

__all__ = ["gaussian_distance", "triangle_distance", "ray_hit_t"]


_ORDERS = {"input": 0, "morton": capi.QK_ORDER_MORTON, "coherent": capi.QK_ORDER_COHERENT}


def _order_flags(order: str, wide: bool) -> int:
    if order not in _ORDERS:
        raise ValueError("order must be 'input', 'morton' or 'coherent'")
    return _ORDERS[order] | (capi.QK_WIDE if wide else 0)


def _tree(kind, items, builder, wide):
    tree = capi.DeviceTree(kind, items, builder=builder)
    if wide:
        tree.build_wide()
    return tree


class _GaussianDistance(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, means, rotations, scales, builder, order, wide):
        items = torch.cat([means, rotations, scales], dim=1).float().contiguous()
        pts = points.float().contiguous()
        tree = _tree("gauss", items, builder, wide)
        res = tree.closest(pts, _order_flags(order, wide))
        d = torch.sqrt(res[:, 0].contiguous().view(torch.float32))
        ctx.tree = tree
        ctx.save_for_backward(pts, res)
        return d

    @staticmethod
    def backward(ctx, grad_d):
        pts, res = ctx.saved_tensors
        gp, gi = ctx.tree.distance_grad(pts, res, grad_d.float().contiguous())
        return gp, gi[:, 0:3], gi[:, 3:7], gi[:, 7:10], None, None, None


class _TriangleDistance(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, vertices, indices, builder, order, wide):
        tris = vertices.float()[indices.long()].reshape(-1, 9).contiguous()
        pts = points.float().contiguous()
        tree = _tree("tri", tris, builder, wide)
        res = tree.closest(pts, _order_flags(order, wide))
        d = torch.sqrt(res[:, 0].contiguous().view(torch.float32))
        ctx.tree = tree
        ctx.nverts = vertices.shape[0]
        ctx.save_for_backward(pts, res, indices)
        return d

    @staticmethod
    def backward(ctx, grad_d):
        pts, res, indices = ctx.saved_tensors
        gp, gv = ctx.tree.distance_grad_vertices(pts, res, indices, ctx.nverts,
                                                 grad_d.float().contiguous())
        return gp, gv, None, None, None, None


class _RayHitT(torch.autograd.Function):
    @staticmethod
    def forward(ctx, origins, dirs, vertices, indices, tmax, builder, order, wide):
        tris = vertices.float()[indices.long()].reshape(-1, 9).contiguous()
        n = origins.shape[0]
        rays = torch.empty((n, 8), dtype=torch.float32, device=origins.device)
        rays[:, 0:3] = origins
        rays[:, 3:6] = dirs
        rays[:, 6] = 1e-6
        rays[:, 7] = tmax
        tree = _tree("tri", tris, builder, wide)
        orders = {"input": 0, "morton": capi.QK_ORDER_MORTON,
                  "direction": capi.QK_ORDER_DIRECTION, "coherent": capi.QK_ORDER_COHERENT}
        if order not in orders:
            raise ValueError("order must be 'input', 'morton', 'direction' or 'coherent'")
        flags = (capi.QK_WIDE if wide else 0) | orders[order]
        out, ids = tree.raycast_ids(rays, flags)
        hit = (out >> 32) != 0
        t = (out & 0xFFFFFFFF).to(torch.int32).view(torch.float32)
        t = torch.where(hit, t, torch.full_like(t, math.inf))
        ctx.tree = tree
        ctx.nverts = vertices.shape[0]
        ctx.save_for_backward(rays, ids, indices)
        ctx.mark_non_differentiable(hit)
        return t, hit

    @staticmethod
    def backward(ctx, grad_t, grad_hit):
        rays, ids, indices = ctx.saved_tensors
        g = torch.where(ids >= 0, grad_t.float(), torch.zeros_like(grad_t, dtype=torch.float32))
        gv, gr = ctx.tree.ray_t_grad_vertices(rays, ids, indices, ctx.nverts, g.contiguous(),
                                              with_rays=True)
        return gr[:, 0:3], gr[:, 3:6], gv, None, None, None, None, None


def gaussian_distance(points, means, rotations, scales, builder: str = "lbvh",
                      order: str = "morton", wide: bool = False):
    """Distance from each point to the nearest solid ellipsoid; differentiable in all inputs.

    points (Q,3), means (N,3), rotations (N,4) xyzw (any norm), scales (N,3) > 0."""
    return _GaussianDistance.apply(points, means, rotations, scales, builder, order, wide)


def triangle_distance(points, vertices, indices, builder: str = "lbvh", order: str = "morton",
                      wide: bool = False):
    """Distance from each point to the nearest triangle of the mesh (vertices (V,3), indices
    (M,3)); differentiable in points and vertices."""
    return _TriangleDistance.apply(points, vertices, indices, builder, order, wide)


def ray_hit_t(origins, dirs, vertices, indices, tmax: float = math.inf, builder: str = "lbvh",
              order: str = "input", wide: bool = False):
    """First-hit distance along each ray (t = inf on a miss) and the hit mask;
    t is differentiable in the vertices, origins and directions."""
    return _RayHitT.apply(origins, dirs, vertices, indices, float(tmax), builder, order, wide)
