"""Seeded synthetic workloads of the engine's benchmark configurations (host side).

The generators live in csrc/scenes.c (exported by libquarry_b200.so) and compute every
transcendental from basic IEEE operations, so a seed yields the same bytes on any host.
bind() points this module at another library exporting the same qs_* functions (a
stand-alone build of scenes.c), so inputs can be made without loading the engine.

Workloads (sizes are the benchmark's; every generator takes smaller sizes for tests):
  terrain   z-up height field on a grid x grid unit lattice, 2 triangles per cell
            (4 sine octaves, amplitudes 8,4,2,1, frequencies 1/64..1/8), 1M downward rays
            from z = +100 and 20k closest-point queries in the bounds padded by 2
  city      131,072 floorless boxes (10 triangles each) on a 363 x 362 lot grid, footprint
            sides U[1,8], log-normal heights (median 10, sigma 0.8); 1M rays from a plane 50
            above the tallest roof with cosine-weighted downward directions; 20k kNN (k=8)
  points    1,048,576 points on a noisy sphere (r=50, radial N(0,0.5)) or uniform in
            [0,100]^3; 20k queries for closest / kNN8 / radius 1.0; a coherent 1% refit
  gaussians 1,048,576 ellipsoids, means U[0,100]^3, log-uniform scales [0.05,1], uniform
            rotations; 262,144 query points
  batch     256 scenes of uneven size: 128 terrains of 1k..500k triangles and 128 uniform
            clouds of 4k..1M points (log-uniform), each with 1k..100k queries split into
            closest / kNN16 / radius (r = 0.02 x diagonal), terrains also with as many rays
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

_P = ctypes.c_void_p
_sig_done = False
_bound = None


def bind(library: ctypes.CDLL) -> None:
    """Use `library` (any build of csrc/scenes.c) for the generators instead of the engine's."""
    global _bound, _sig_done
    _bound = library
    _sig_done = False


def _lib():
    global _sig_done
    if _bound is not None:
        L = _bound
    else:
        from . import capi

        L = capi.lib()
    if not _sig_done:
        L.qs_cfg_terrain.restype = ctypes.c_int64
        L.qs_cfg_terrain.argtypes = [ctypes.c_int, ctypes.c_uint64, _P]
        L.qs_cfg_down_rays.restype = None
        L.qs_cfg_down_rays.argtypes = [ctypes.c_int] + [ctypes.c_float] * 5 + [ctypes.c_uint64, _P]
        L.qs_cfg_cosine_rays.restype = None
        L.qs_cfg_cosine_rays.argtypes = [ctypes.c_int] + [ctypes.c_float] * 5 + [ctypes.c_uint64, _P]
        L.qs_cfg_uniform_points.restype = None
        L.qs_cfg_uniform_points.argtypes = [ctypes.c_int, _P, _P, ctypes.c_uint64, ctypes.c_uint64, _P]
        L.qs_cfg_city.restype = ctypes.c_int64
        L.qs_cfg_city.argtypes = [ctypes.c_int, ctypes.c_uint64, _P, _P]
        L.qs_cfg_points.restype = None
        L.qs_cfg_points.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, _P]
        L.qs_cfg_coherent_motion.restype = None
        L.qs_cfg_coherent_motion.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                             ctypes.c_uint64, _P, _P]
        L.qs_cfg_gaussians.restype = None
        L.qs_cfg_gaussians.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_uint64, _P]
        L.qs_log_uniform_int.restype = ctypes.c_int
        L.qs_log_uniform_int.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.qs_demo_mesh.restype = ctypes.c_int64
        L.qs_demo_mesh.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                   ctypes.c_int, _P]
        L.qs_demo_gaussians.restype = None
        L.qs_demo_gaussians.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, _P]
        for f in ("qs_det_sin", "qs_det_cos", "qs_det_log", "qs_det_exp"):
            getattr(L, f).restype = ctypes.c_double
            getattr(L, f).argtypes = [ctypes.c_double]
        _sig_done = True
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(_P)


def bounds_of(tris: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    v = tris.reshape(-1, 3)
    return v.min(axis=0), v.max(axis=0)


def terrain(grid: int = 256, seed: int = 1) -> np.ndarray:
    L = _lib()
    n = L.qs_cfg_terrain(grid, seed, None)
    t = np.zeros((n, 9), np.float32)
    L.qs_cfg_terrain(grid, seed, _p(t))
    return t


def down_rays(count: int, x0: float, x1: float, y0: float, y1: float, z: float,
              seed: int = 1) -> np.ndarray:
    r = np.zeros((count, 8), np.float32)
    _lib().qs_cfg_down_rays(count, x0, x1, y0, y1, z, seed, _p(r))
    return r


def cosine_rays(count: int, x0: float, x1: float, y0: float, y1: float, z: float,
                seed: int = 1) -> np.ndarray:
    r = np.zeros((count, 8), np.float32)
    _lib().qs_cfg_cosine_rays(count, x0, x1, y0, y1, z, seed, _p(r))
    return r


def uniform_points(count: int, lo, hi, seed: int = 1, stream: int = 13) -> np.ndarray:
    lo = np.ascontiguousarray(lo, np.float32)
    hi = np.ascontiguousarray(hi, np.float32)
    p = np.zeros((count, 3), np.float32)
    _lib().qs_cfg_uniform_points(count, _p(lo), _p(hi), seed, stream, _p(p))
    return p


def city(buildings: int = 131072, seed: int = 1) -> tuple[np.ndarray, float]:
    L = _lib()
    n = L.qs_cfg_city(buildings, seed, None, None)
    t = np.zeros((n, 9), np.float32)
    top = ctypes.c_float(0.0)
    L.qs_cfg_city(buildings, seed, _p(t), ctypes.byref(top))
    return t, top.value


def point_cloud(kind: str = "volume", count: int = 1048576, seed: int = 1) -> np.ndarray:
    p = np.zeros((count, 3), np.float32)
    _lib().qs_cfg_points(1 if kind == "volume" else 0, count, seed, _p(p))
    return p


def coherent_motion(pts: np.ndarray, fraction: float = 0.01, sigma: float = 0.05,
                    seed: int = 1) -> tuple[np.ndarray, np.ndarray]:
    pts = np.ascontiguousarray(pts, np.float32)
    dirty = max(1, int(round(fraction * pts.shape[0])))
    out = np.zeros_like(pts)
    ids = np.zeros(dirty, np.int32)
    _lib().qs_cfg_coherent_motion(_p(pts), pts.shape[0], dirty, sigma, seed, _p(out), _p(ids))
    return out, ids


def gaussians(count: int = 1048576, smin: float = 0.05, smax: float = 1.0,
              seed: int = 1) -> np.ndarray:
    g = np.zeros((count, 10), np.float32)
    _lib().qs_cfg_gaussians(count, smin, smax, seed, _p(g))
    return g


def log_uniform_int(seed: int, stream: int, lo: int, hi: int) -> int:
    return _lib().qs_log_uniform_int(seed, stream, lo, hi)


def demo_mesh_tris(kind: int, grid: int, random_tris: int, seed: int, buildings: int) -> np.ndarray:
    L = _lib()
    n = L.qs_demo_mesh(kind, grid, random_tris, seed, buildings, None)
    if n < 0:
        raise ValueError("unknown demo mesh kind")
    t = np.zeros((n, 9), np.float32)
    L.qs_demo_mesh(kind, grid, random_tris, seed, buildings, _p(t))
    return t


def demo_gaussians(kind: int, count: int, seed: int) -> np.ndarray:
    g = np.zeros((count, 10), np.float32)
    _lib().qs_demo_gaussians(kind, count, seed, _p(g))
    return g


# ---------------------------------------------------------------------------------------
# the benchmark configurations
# ---------------------------------------------------------------------------------------
@dataclass
class TerrainConfig:
    tris: np.ndarray
    rays: np.ndarray
    queries: np.ndarray


def terrain_config(grid: int = 256, rays: int = 1_000_000, queries: int = 20_000,
                   seed: int = 1) -> TerrainConfig:
    tris = terrain(grid, seed)
    lo, hi = bounds_of(tris)
    r = down_rays(rays, 0.0, float(grid), 0.0, float(grid), 100.0, seed)
    q = uniform_points(queries, lo - 2.0, hi + 2.0, seed, 13)
    return TerrainConfig(tris, r, q)


@dataclass
class CityConfig:
    tris: np.ndarray
    rays: np.ndarray
    queries: np.ndarray
    top: float


def city_config(buildings: int = 131072, rays: int = 1_000_000, queries: int = 20_000,
                seed: int = 1) -> CityConfig:
    tris, top = city(buildings, seed)
    lo, hi = bounds_of(tris)
    r = cosine_rays(rays, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]), top + 50.0,
                    seed)
    q = uniform_points(queries, lo, hi, seed, 13)
    return CityConfig(tris, r, q, top)


@dataclass
class BatchScene:
    """One scene of the batched workload: primitives and its four query sets."""
    kind: str              # "tri" (terrain) or "point" (uniform cloud)
    items: np.ndarray      # (n, 9) triangles or (n, 3) points
    closest: np.ndarray    # (q1, 3)
    knn: np.ndarray        # (q2, 3)
    radius: np.ndarray     # (q3, 3)
    r: float               # 0.02 x the scene's bounding-box diagonal
    rays: np.ndarray       # (q, 8) downward rays (terrain scenes), (0, 8) otherwise


@dataclass
class BatchConfig:
    terrains: list
    clouds: list
    k: int


def batch_scene_sizes(index: int, prim_range: tuple[int, int],
                      query_range: tuple[int, int], first_seed: int = 1000) -> tuple[int, int]:
    """Primitive and query counts of scene `index` (seed first_seed + index, log-uniform)."""
    seed = first_seed + index
    return (log_uniform_int(seed, 1, prim_range[0], prim_range[1]),
            log_uniform_int(seed, 2, query_range[0], query_range[1]))


def batch_config(terrains: int = 128, clouds: int = 128,
                 tri_range: tuple[int, int] = (1_000, 500_000),
                 point_range: tuple[int, int] = (4_000, 1_000_000),
                 query_range: tuple[int, int] = (1_000, 100_000), k: int = 16,
                 first_seed: int = 1000) -> BatchConfig:
    """The batched uneven workload: `terrains` height-field meshes (scenes 0..terrains-1) and
    `clouds` uniform point clouds (the following scene indices).  Scene i uses seed
    first_seed + i;
    its Q queries are uniform in its bounds, the first third closest, the next third kNN, the
    rest radius at r = 0.02 x diagonal; terrain scenes also get Q rays straight down from
    z = +100."""
    out_t, out_c = [], []
    for i in range(terrains + clouds):
        is_tri = i < terrains
        n, q = batch_scene_sizes(i, tri_range if is_tri else point_range, query_range,
                                 first_seed)
        seed = first_seed + i
        if is_tri:
            grid = max(2, int(round((n / 2) ** 0.5)))
            items = terrain(grid, seed)
            lo, hi = bounds_of(items)
        else:
            items = point_cloud("volume", n, seed)
            lo, hi = items.min(axis=0), items.max(axis=0)
        pts = uniform_points(q, lo, hi, seed, 13)
        a, b = q // 3, 2 * (q // 3)
        diag = float(np.sqrt(np.sum((hi.astype(np.float64) - lo.astype(np.float64)) ** 2)))
        r = float(np.float32(0.02 * diag))
        if is_tri:
            rays = down_rays(q, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]), 100.0, seed)
        else:
            rays = np.zeros((0, 8), np.float32)
        sc = BatchScene("tri" if is_tri else "point", items, pts[:a], pts[a:b], pts[b:], r, rays)
        (out_t if is_tri else out_c).append(sc)
    return BatchConfig(out_t, out_c, k)


def _centroids(items: np.ndarray) -> np.ndarray:
    if items.shape[1] == 9:
        return items.reshape(-1, 3, 3).mean(axis=1)
    return items[:, :3]


def topology_edit(items: np.ndarray, fraction: float = 0.01, mode: str = "cluster",
                  seed: int = 1):
    """A GpuTopoEdit script over `items` (n, stride) touching `fraction` of them: a quarter
    deleted, a quarter inserted at random new indices, a quarter appended, a quarter moved.
    "cluster" draws every touched primitive from the ones nearest a random anchor (and new
    primitives as shifted copies of them); "scatter" draws them uniformly.  Returns (new scene,
    deleted old indices, inserted new indices, moved new indices), index arrays ascending."""
    rng = np.random.default_rng(seed)
    items = np.ascontiguousarray(items, np.float32)
    n = items.shape[0]
    q = max(1, int(round(fraction * n / 4)))
    cen = _centroids(items)
    if mode == "cluster":
        anchor = cen[rng.integers(n)]
        pool = np.argsort(((cen - anchor) ** 2).sum(axis=1), kind="stable")[: 4 * q]
    elif mode == "scatter":
        pool = np.arange(n)
    else:
        raise ValueError("mode must be 'cluster' or 'scatter'")
    deleted = np.sort(rng.choice(pool, q, replace=False)).astype(np.int32)
    ext = 0.05 * float(np.linalg.norm(cen.max(axis=0) - cen.min(axis=0))) / max(n, 1) ** (1 / 3)

    def fresh(count):
        src = items[rng.choice(pool, count)].copy()
        shift = rng.normal(0.0, ext, (count, 3)).astype(np.float32)
        if items.shape[1] == 9:
            src += np.tile(shift, 3)
        else:
            src[:, :3] += shift
        return src

    survivors = np.delete(items, deleted, axis=0)
    n_new = n - q + 2 * q
    tail = n_new - q
    inserted = np.sort(rng.choice(tail, q, replace=False)).astype(np.int32)
    new = np.empty((n_new, items.shape[1]), np.float32)
    keep = np.ones(tail, bool)
    keep[inserted] = False
    new[:tail][keep] = survivors
    new[inserted] = fresh(q)
    new[tail:] = fresh(q)
    # moved: survivors from the pool, at their new indices
    old_to_new = np.full(n, -1, np.int64)
    old_to_new[np.setdiff1d(np.arange(n), deleted)] = np.flatnonzero(keep)
    cand = old_to_new[np.setdiff1d(pool, deleted)]
    moved = np.sort(rng.choice(cand, min(q, cand.size), replace=False)).astype(np.int32)
    shift = rng.normal(0.0, ext, (moved.size, 3)).astype(np.float32)
    if items.shape[1] == 9:
        new[moved] += np.tile(shift, 3)
    else:
        new[moved, :3] += shift
    return new, deleted, inserted, moved
