"""FP64 restatements of the differentiated leaf tests.  TEST INFRASTRUCTURE ONLY.

The engine's adjoint kernels (quarry-gpu_b200/csrc/qk_grad.cu) return gradients of
  * the distance from a query point to its selected Gaussian's solid ellipsoid
    (quarry's gaussianDist2, src/core/gaussian.h:66-131, taken as a distance, not squared),
  * the distance from a query point to its selected triangle (closestPointOnTriangle,
    src/core/geometry.h:198-259),
  * the first-hit t of a ray on its selected triangle (intersectTriangle,
    src/core/geometry.h:112-176).
quarry has no backward pass, so these are checked against (1) central finite differences of
the FP64 functions below with the forward's selection held fixed, and (2) analytic FP64
gradients written from the geometry: the envelope theorem for the distances (the gradient of
a minimum distance is the unit vector from the closest point, propagated through the frame
and the ellipsoid's shape), and the plane-crossing derivative for t.  Only tests/ and
bench.py's checks import this module.
"""
from __future__ import annotations

import numpy as np

H = 1e-3  # finite-difference step of the checks


# ---------------------------------------------------------------------------------------
# Gaussians: frame, distance, analytic gradients
# ---------------------------------------------------------------------------------------
def quat_axes(q):
    """Rotation axes (u, v, w) of quaternions q (..., 4) in xyzw order, normalised first
    (gaussianAxes, src/core/gaussian.h:23-45)."""
    q = q / np.linalg.norm(q, axis=-1, keepdims=True)
    x, y, z, w = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    u = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y + z * w), 2 * (x * z - y * w)], -1)
    v = np.stack([2 * (x * y - z * w), 1 - 2 * (x * x + z * z), 2 * (y * z + x * w)], -1)
    t = np.stack([2 * (x * z + y * w), 2 * (y * z - x * w), 1 - 2 * (x * x + y * y)], -1)
    return u, v, t


def ellipsoid_d(p, g, iters: int = 200):
    """Distance from points p (K,3) to the solid ellipsoids g (K,10) = mean, quat xyzw,
    scales, in FP64.  The closest surface point in the local frame is x = s^2 y / (t + s^2)
    with t the root of sum (s y / (t + s^2))^2 = 1 (Eberly), found by bisection on
    [0, 2 max(s) |y|] (iters halvings).  Returns (d, y, x, s, (u, v, w), p - mean);
    d = 0 inside."""
    u, v, w = quat_axes(g[:, 3:7])
    dp = p - g[:, 0:3]
    y = np.stack([(dp * u).sum(-1), (dp * v).sum(-1), (dp * w).sum(-1)], -1)
    s = g[:, 7:10]
    inside = ((y / s) ** 2).sum(-1) <= 1.0
    lo = np.zeros(len(p))
    hi = 2 * s.max(-1) * np.linalg.norm(y, axis=-1)
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        f = ((s * y / (mid[:, None] + s * s)) ** 2).sum(-1) - 1
        lo = np.where(f > 0, mid, lo)
        hi = np.where(f > 0, hi, mid)
    t = 0.5 * (lo + hi)
    x = s * s * y / (t[:, None] + s * s)
    d = np.where(inside, 0.0, np.linalg.norm(y - x, axis=-1))
    return d, y, x, s, (u, v, w), dp


def quat_grad(q, dp, nl):
    """d(nl . y)/dq for y = (u.dp, v.dp, w.dp), axes from the normalised quaternion q (K,4)
    xyzw, nl (K,3) held fixed: the derivatives of the axis formulas with respect to the unit
    quaternion's components, projected through the normalisation
    (d qhat / dq = (I - qhat qhat^T) / |q|)."""
    norm = np.linalg.norm(q, axis=-1, keepdims=True)
    qh = q / norm
    x, y, z, w = qh[:, 0], qh[:, 1], qh[:, 2], qh[:, 3]
    zero = np.zeros_like(x)

    def vec(a, b, c):
        return np.stack([a, b, c], -1)

    # d axis / d (x, y, z, w) for u, v, w (the third axis is called t here)
    du = [vec(zero, 2 * y, 2 * z), vec(-4 * y, 2 * x, -2 * w), vec(-4 * z, 2 * w, 2 * x),
          vec(zero, 2 * z, -2 * y)]
    dv = [vec(2 * y, -4 * x, 2 * w), vec(2 * x, zero, 2 * z), vec(-2 * w, -4 * z, 2 * y),
          vec(-2 * z, zero, 2 * x)]
    dt = [vec(2 * z, -2 * w, -4 * x), vec(2 * w, 2 * z, -4 * y), vec(2 * x, 2 * y, zero),
          vec(2 * y, -2 * x, zero)]
    gh = np.stack([nl[:, 0] * (du[j] * dp).sum(-1) + nl[:, 1] * (dv[j] * dp).sum(-1) +
                   nl[:, 2] * (dt[j] * dp).sum(-1) for j in range(4)], -1)
    return (gh - qh * (qh * gh).sum(-1, keepdims=True)) / norm


def gaussian_analytic(P, G, ids, iters: int = 200):
    """Analytic FP64 gradients of L = sum_i d_i for query points P (Q,3) on Gaussians G
    (N,10), query i selecting Gaussian ids[i] (all >= 0).  Returns (d, dL/dP (Q,3),
    dL/dG (N,10) summed per Gaussian: mean, quat, scale)."""
    dd, y, x, s, (u, v, w), dp = ellipsoid_d(P, G[ids], iters)
    out = dd > 0
    nl = np.zeros_like(y)
    nl[out] = (y[out] - x[out]) / dd[out, None]
    nw = nl[:, 0:1] * u + nl[:, 1:2] * v + nl[:, 2:3] * w
    gq = quat_grad(G[ids, 3:7], dp, nl)
    per = np.concatenate([-nw, gq, -nl * x / s], axis=1)
    gG = np.zeros((G.shape[0], 10))
    np.add.at(gG, ids, per)
    return dd, nw, gG


# ---------------------------------------------------------------------------------------
# triangles: closest point and ray t
# ---------------------------------------------------------------------------------------
def closest_tri(p, a, b, c):
    """Vectorised Ericson closest point on triangles (a, b, c) in FP64, the region order of
    closestPointOnTriangle (src/core/geometry.h:198-259); returns (q, wa, wb, wc)."""
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = (ab * ap).sum(-1), (ac * ap).sum(-1)
    bp = p - b
    d3, d4 = (ab * bp).sum(-1), (ac * bp).sum(-1)
    cp = p - c
    d5, d6 = (ab * cp).sum(-1), (ac * cp).sum(-1)
    vc = d1 * d4 - d3 * d2
    vb = d5 * d2 - d1 * d6
    va = d3 * d6 - d5 * d4
    wb = np.zeros(len(p))
    wc = np.zeros(len(p))
    done = np.zeros(len(p), bool)

    def put(mask, b_, c_):
        nonlocal done
        m = mask & ~done
        wb[m] = b_[m] if np.ndim(b_) else b_
        wc[m] = c_[m] if np.ndim(c_) else c_
        done |= m

    with np.errstate(divide="ignore", invalid="ignore"):
        put((d1 <= 0) & (d2 <= 0), 0.0, 0.0)
        put((d3 >= 0) & (d4 <= d3), 1.0, 0.0)
        put((vc <= 0) & (d1 >= 0) & (d3 <= 0), d1 / (d1 - d3), np.zeros(len(p)))
        put((d6 >= 0) & (d5 <= d6), 0.0, 1.0)
        put((vb <= 0) & (d2 >= 0) & (d6 <= 0), np.zeros(len(p)), d2 / (d2 - d6))
        tbc = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        put((va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0), 1.0 - tbc, tbc)
        den = va + vb + vc
        put(np.ones(len(p), bool), vb / den, vc / den)
    wa = 1 - wb - wc
    q = a * wa[:, None] + b * wb[:, None] + c * wc[:, None]
    return q, wa, wb, wc


def ray_t(o, d, a, b, c):
    """t where the rays o + t d cross the planes of triangles (a, b, c), FP64."""
    n = np.cross(b - a, c - a)
    return ((n * (a - o)).sum(-1)) / ((n * d).sum(-1))


def ray_analytic(O, D, a, b, c):
    """Analytic FP64 derivative of t with respect to the three vertices (each (K,3)) and the
    ray origin / direction: with k = n / (n . d), dt/da_j = w_j k (w the barycentric weights
    of the hit point), dt/do = -k, dt/dd = -t k."""
    tt = ray_t(O, D, a, b, c)
    nrm = np.cross(b - a, c - a)
    nd = (nrm * D).sum(-1)
    h = O + D * tt[:, None]
    nn = (nrm * nrm).sum(-1)
    u = (np.cross(h - a, c - a) * nrm).sum(-1) / nn
    v = (np.cross(b - a, h - a) * nrm).sum(-1) / nn
    k = nrm / nd[:, None]
    return tt, (1 - u - v, u, v), k


def rel_err(g, ref, floor):
    """|g - ref| / max(|ref|, floor), elementwise."""
    return np.abs(g - ref) / np.maximum(np.abs(ref), floor)


def fd_stats(errs) -> dict:
    errs = np.asarray(errs, dtype=np.float64)
    return {"median": float(np.median(errs)), "p99": float(np.percentile(errs, 99)),
            "max": float(errs.max()), "count": int(errs.size)}


def central(loss, h: float = H) -> tuple[float, float]:
    """(central difference at h, Richardson extrapolation (4 D(h/2) - D(h)) / 3, which cancels
    the difference's h^2 truncation term)."""
    fd = (loss(h) - loss(-h)) / (2 * h)
    fd2 = (loss(h / 2) - loss(-h / 2)) / h
    return fd, (4 * fd2 - fd) / 3
