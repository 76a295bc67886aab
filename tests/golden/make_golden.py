"""Regenerates tests/golden/*.npz from quarry's own CPU reference.

Needs oracle/_ref/libquarry_ref.so (quarry's src/core + src/cpu sources compiled where they
lie by oracle/Makefile, which reads them from /root/reference).  Each fixture stores the
inputs and the reference's outputs for one primitive kind:

    python tests/golden/make_golden.py

Inputs come from quarry.workloads (deterministic bytes on every host), so the fixtures only
need regenerating if the generators change.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "quarry-gpu_b200"))

import oracle  # noqa: E402
from quarry import workloads  # noqa: E402

OUT = Path(__file__).resolve().parent


def rays_for(lo, hi, n, seed):
    rng = np.random.default_rng(seed)
    c = (lo + hi) / 2
    ext = hi - lo
    rad = 1.6 * float(np.linalg.norm(ext))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = c + d * rad
    tgt = c + (rng.random((n, 3)) * 2 - 1) * ext * 0.9
    dirs = tgt - o
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3], r[:, 3:6], r[:, 6], r[:, 7] = o, dirs, 1e-6, rad * 4
    down = workloads.down_rays(n, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                               float(hi[2]) + 5.0, seed)
    return np.concatenate([r, down])


def main():
    R = oracle.Reference()
    assert R.selftest()
    cases = {
        "tri": workloads.demo_mesh_tris(2, 12, 300, 7, 0),
        "city": workloads.city(60, 3)[0],
        "point": workloads.point_cloud("sphere", 4000, 3),
        "gauss": workloads.gaussians(1500, 0.05, 1.0, 3),
    }
    for name, items in cases.items():
        kind = "tri" if name in ("tri", "city") else name
        if kind == "tri":
            lo, hi = workloads.bounds_of(items)
        else:
            lo, hi = items[:, :3].min(0), items[:, :3].max(0)
        q = workloads.uniform_points(600, lo - 1, hi + 1, 5, 21)
        data = {"items": items, "queries": q}
        closest, _, _ = R.closest(kind, items, q)
        knn8, _, _ = R.knn(kind, items, q, 8)
        r = {"tri": 2.0, "point": 3.0, "gauss": 1.0}[kind]
        off, keys, _ = R.radius(kind, items, q, r)
        data.update(closest=closest, knn8=knn8, radius=np.float32(r), radius_offsets=off,
                    radius_keys=keys)
        if kind == "tri":
            rays = rays_for(lo, hi, 800, 9)
            hits, _, _ = R.raycast(items, rays)
            data.update(rays=rays, ray_results=hits)
        np.savez_compressed(OUT / f"{name}.npz", **data)
        print(name, {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main()
