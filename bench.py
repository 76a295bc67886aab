"""Benchmark of the B200 spatial-query engine on the city workload.

Workload (one GPU): 131,072 floorless box buildings (1,310,720 triangles) on a 363 x 362 lot
grid, 1,000,000 rays from a plane 50 units above the tallest roof with cosine-weighted
downward directions, 20,000 kNN (k=8) queries uniform in the scene bounds.  Seeded synthetic
inputs generated by quarry.workloads (same bytes on every host).

A step is one pass of the hot path over the resident inputs: trace the 1M rays (Morton
order) through the tree.  `value` is rays per second over the timed steps (device time,
CUDA events, L2 flushed between steps), `e2e` the same through the C ABI from pinned host
buffers with the 32 MB ray upload and 8 MB result read-back inside the timed region.  The
kNN pass and the build are timed beside it.  Every variant's results are compared bit for
bit with each other, and the timed variant with quarry's own CPU reference on a sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload city|terrain] [--small]

Multi-GPU: one process per GPU (torchrun); every rank builds its own replica of the scene
and traces its own 1M rays (weak scaling, no data-path collective); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "quarry-gpu_b200"))

METRIC = ("Mrays/s, Mqueries/s at bit-exact hash; batched vs per-scene loop; bwd/fwd ratio")
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 400; 20 for --workload batch)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="city", choices=["city", "terrain", "grad", "batch", "points"])
    ap.add_argument("--tune-cache", default=None, help="autotuner JSON (default: user cache)")
    ap.add_argument("--retune", action="store_true", help="ignore cached autotuner choices")
    ap.add_argument("--small", action="store_true", help="small inputs (profiling captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", default="", help="time only this variant (profiling)")
    ap.add_argument("--dump", default="", help="also write the inputs as QRYD / QRCD files "
                                                "into this directory (for other engines)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.workload == "batch" else 400
    return args


def profiled_traffic(workload: str, variant: str):
    """DRAM bytes of one launch of this variant's kernel from the ncu summary in profiles/."""
    p = ROOT / "profiles" / "traffic.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) >= 4 and cells[0] == workload and cells[1] == variant and cells[3].isdigit():
            return int(cells[3])
    return None


def peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return PEAKS_FALLBACK, "fallback"


def coherent_order(rays: np.ndarray) -> np.ndarray:
    """The engine's coherent ray order (QK_ORDER_COHERENT), recomputed on the host: a Morton
    key over origin and direction, the non-flat axes (bounds of 4,096 rays spaced count /
    4,096 apart) with b bits each, b * axes <= log2(bucket count), the bucket count at most
    32,768 and count / 4; ties keep input order."""
    n = rays.shape[0]
    kb = 4
    while (2 << kb) <= 32768 and (2 << kb) <= n // 4:
        kb += 1
    x = rays[:, :6].astype(np.float32)
    samples = min(n, 4096)
    pick = x[np.arange(samples, dtype=np.int64) * (n // samples)]
    lo, hi = pick.min(0), pick.max(0)
    ext = hi - lo
    live = [a for a in range(6) if ext[a] > 0 and np.isfinite(ext[a])]
    if not live:
        return np.arange(n)
    bits = min(kb // len(live), 10)
    q = [np.clip((x[:, a] - lo[a]) * np.float32((1 << bits) / ext[a]), 0,
                 (1 << bits) - 1).astype(np.uint32) for a in live]
    key = np.zeros(n, np.uint32)
    for bit in range(bits - 1, -1, -1):
        for qa in q:
            key = (key << np.uint32(1)) | ((qa >> np.uint32(bit)) & np.uint32(1))
    return np.argsort(key, kind="stable")


def make_workload(name: str, small: bool, rank: int):
    from quarry import workloads as w

    seed = 1 + rank  # each rank traces its own rays over its own replica of the same scene
    if name == "city":
        b = 4096 if small else 131072
        nr = 100_000 if small else 1_000_000
        cfg = w.city_config(b, nr, 20_000, 1)
        if rank:
            lo, hi = w.bounds_of(cfg.tris)
            cfg.rays = w.cosine_rays(nr, float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]),
                                     cfg.top + 50.0, seed)
        desc = {"workload": "city", "buildings": b, "triangles": int(cfg.tris.shape[0]),
                "rays": nr, "knn_queries": 20_000, "k": 8}
    else:
        g = 64 if small else 256
        nr = 100_000 if small else 1_000_000
        cfg = w.terrain_config(g, nr, 20_000, seed)
        desc = {"workload": "terrain", "grid": g, "triangles": int(cfg.tris.shape[0]),
                "rays": nr, "closest_queries": 20_000}
    return cfg, desc


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"qk_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            # start timing only once the sampler is producing lines
            deadline = time.time() + 10.0
            while time.time() < deadline and self.path.stat().st_size == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict:
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


_RANKS = None


def init_dist(args):
    """One process per GPU over NCCL (quarry.dist); world 1 needs no process group."""
    global _RANKS
    from quarry import dist

    _RANKS = dist.init(backend="nccl" if int(os.environ.get("WORLD_SIZE", "1")) > 1 else None)
    return _RANKS.world, _RANKS.rank, _RANKS.local


def barrier(world):
    from quarry import dist

    if _RANKS is not None:
        dist.barrier(_RANKS)


def max_over_ranks(world, value: float) -> float:
    from quarry import dist

    return dist.max_over_ranks(_RANKS, value) if _RANKS is not None else float(value)


# ---------------------------------------------------------------------------------------
# CPU reference (quarry's own CPU code, compiled from its sources into oracle/_ref)
# ---------------------------------------------------------------------------------------
def cpu_reference_rays(tris, rays, threads: int):
    import oracle

    if oracle.REF_PATH.exists():
        R = oracle.Reference()
        out, ms, build_ms = R.raycast(tris, rays, threads)
        return out, ms, build_ms, "reference"
    # the oracle port when the reference could not be compiled on this machine
    ref = oracle.LBVH("tri", tris)
    t0 = time.perf_counter()
    out = ref.raycast(rays, threads)
    return out, (time.perf_counter() - t0) * 1e3, 0.0, "port"


def reference_arm(args, world, rank):
    """--impl reference: time quarry's CPU reference on the host cores (rank 0 only)."""
    if rank != 0:
        return
    cfg, desc = make_workload(args.workload, args.small, 0)
    threads = os.cpu_count() or 1
    sample = min(len(cfg.rays), 200_000 if not args.small else 50_000)
    rays = cfg.rays[:sample]
    times = []
    kind = "reference"
    for i in range(args.warmup + args.steps):
        _, ms, _, kind = cpu_reference_rays(cfg.tris, rays, threads)
        if i >= args.warmup:
            times.append(ms)
    ms = float(np.mean(times))
    value = sample / (ms * 1e-3) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
            "config": desc,
            "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads,
                             "kind": kind,
                             "sample": f"first {sample} of the workload's rays per step, "
                                       f"reference BVH built once per step (build excluded)"},
            "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# differentiable queries: forward and forward + backward time
# ---------------------------------------------------------------------------------------
def grad_arm(args, world, rank, local):
    """1,048,576 Gaussians (means U[0,100]^3, log-uniform scales [0.05, 1], random rotations)
    with 262,144 query points, loss = sum of point-to-ellipsoid distances; and 1M downward
    rays on the 256 x 256 terrain, loss = sum of first-hit t, gradients to the vertices."""
    import torch

    from quarry import capi, workloads as w

    torch.cuda.set_device(local)
    small = args.small
    ng, nq = (65_536, 16_384) if small else (1_048_576, 262_144)
    g = torch.tensor(w.gaussians(ng, 0.05, 1.0, 1 + rank), device="cuda")
    q = torch.tensor(w.uniform_points(nq, [0, 0, 0], [100, 100, 100], 1 + rank, 31), device="cuda")
    flags = capi.QK_ORDER_MORTON
    l2 = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def timed(fn, steps):
        for _ in range(3):
            fn()
        ts = []
        for _ in range(steps):
            l2.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    state = {}

    def g_build():
        state["tree"] = capi.DeviceTree("gauss", g)

    def g_fwd():
        res = state["tree"].closest(q, flags)
        state["res"] = res
        state["d"] = torch.sqrt(res[:, 0].contiguous().view(torch.float32))

    def g_bwd():
        state["grads"] = state["tree"].distance_grad(q, state["res"])

    g_build()
    build_ms = timed(g_build, 5)
    # forward schedule: every variant returns the same bits; the fastest is timed
    state["tree"].build_wide()
    fwd_variants = {"morton": capi.QK_ORDER_MORTON, "input": 0,
                    "split_morton": capi.QK_ORDER_MORTON | capi.QK_TUNE_SPLIT,
                    "wide_morton": capi.QK_ORDER_MORTON | capi.QK_WIDE,
                    "coherent": capi.QK_ORDER_COHERENT,
                    "wide_coherent": capi.QK_ORDER_COHERENT | capi.QK_WIDE}
    base = state["tree"].closest(q, 0).clone()
    fwd_by = {}
    for name, f in fwd_variants.items():
        if not torch.equal(state["tree"].closest(q, f), base):
            raise RuntimeError(f"Gaussian closest variant {name} differs")
        flags = f
        fwd_by[name] = timed(g_fwd, 5)
    fwd_variant = min(fwd_by, key=fwd_by.get)
    flags = fwd_variants[fwd_variant]
    fwd_ms = timed(g_fwd, 10)
    bwd_ms = timed(g_bwd, 10)

    # triangles: 1M down rays on the terrain, loss = sum of t
    tris = w.terrain(64 if small else 256, 1)
    nr = 100_000 if small else 1_000_000
    grid = 64 if small else 256
    rays = capi.to_device(w.down_rays(nr, 0.0, float(grid), 0.0, float(grid), 100.0, 1), np.float32)
    tri_tree = capi.DeviceTree("tri", tris)

    ray_flags = {"morton": capi.QK_ORDER_MORTON, "coherent": capi.QK_ORDER_COHERENT}
    state["rflags"] = capi.QK_ORDER_MORTON

    def r_fwd():
        state["out"], state["ids"] = tri_tree.raycast_ids(rays, state["rflags"])

    def r_bwd():
        state["rg"] = tri_tree.ray_t_grad(rays, state["ids"], None, with_rays=False)

    # the ray order is chosen by measurement too (same hits and ids for both)
    r_by, r_base = {}, None
    for name, f in ray_flags.items():
        state["rflags"] = f
        r_fwd()
        got = (state["out"].clone(), state["ids"].clone())
        if r_base is None:
            r_base = got
        elif not (torch.equal(got[0], r_base[0]) and torch.equal(got[1], r_base[1])):
            raise RuntimeError(f"ray order {name} differs")
        r_by[name] = timed(r_fwd, 5)
    ray_order = min(r_by, key=r_by.get)
    state["rflags"] = ray_flags[ray_order]
    r_fwd()
    rf_ms = timed(r_fwd, 10)
    rb_ms = timed(r_bwd, 10)
    if rank == 0:
        line = {"metric": METRIC, "value": round((fwd_ms + bwd_ms) / fwd_ms, 4),
                "unit": "fwd+bwd / fwd (Gaussian closest distance)", "n_gpus": world,
                "steps": 10, "warmup": 3, "ms_per_step": round(fwd_ms + bwd_ms, 4),
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 forward, f64 adjoint", "data": "synthetic (seeded generators)",
                "config": {"workload": "gaussian distance + ray t gradients", "gaussians": ng,
                           "queries": nq, "rays": nr, "terrain_grid": grid,
                           "order": "fastest of the variants below",
                           "l2": "flushed between timed steps"},
                "gaussian": {"build_ms": round(build_ms, 3), "forward_ms": round(fwd_ms, 4),
                             "forward_variant": fwd_variant,
                             "forward_variants_ms": {k: round(v, 4) for k, v in fwd_by.items()},
                             "backward_ms": round(bwd_ms, 4),
                             "fwd_bwd_over_fwd": round((fwd_ms + bwd_ms) / fwd_ms, 4),
                             "mqueries_per_s": round(nq / (fwd_ms * 1e-3) / 1e6, 2)},
                "rays": {"forward_ms": round(rf_ms, 4), "backward_ms": round(rb_ms, 4),
                         "order": ray_order,
                         "forward_orders_ms": {k: round(v, 4) for k, v in r_by.items()},
                         "fwd_bwd_over_fwd": round((rf_ms + rb_ms) / rf_ms, 4)}}
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# topology edits: subtree surgery against a rebuild of the edited scene
# ---------------------------------------------------------------------------------------
def topology_timing(kind, items, builder, bins, queries_d, seed, timed_ms, rays_d=None):
    """1% edits of quarry's GpuTopoEdit kind (a quarter each deleted, inserted, appended and
    moved), "cluster" (around one spot) and "scatter" (uniform): qk_update_topology on the
    built tree against qk_build of the edited scene, both device-timed with the scripts
    already resident.  The edited tree must answer closest / kNN (and rays) like the rebuild."""
    import ctypes

    import torch

    from quarry import capi, workloads as w

    out = {}
    for mode in ("cluster", "scatter"):
        new, dele, ins, mov = w.topology_edit(items, 0.01, mode, seed)
        base = capi.DeviceTree(kind, items, builder=builder, sah_bins=bins)
        n_new = len(new)
        new_d = capi.to_device(new, np.float32)
        dele_d, ins_d, mov_d = (capi.to_device(a, np.int32) for a in (dele, ins, mov))
        app = n_new - len(items) + len(dele) - len(ins)
        tail = torch.arange(n_new - app, n_new, device="cuda")
        extra = new_d[torch.cat([ins_d.long(), tail])].contiguous()
        moved_items = new_d[mov_d.long()].contiguous()
        e = capi.QkTopoEdit(dele_d.data_ptr(), len(dele), ins_d.data_ptr(), len(ins), app,
                            mov_d.data_ptr(), len(mov), extra.data_ptr(), moved_items.data_ptr())
        arrays, nt = base._alloc(n_new)
        nb = capi.lib().qk_update_workspace_bytes(base.kind, base.n, n_new, int(extra.shape[0]))
        ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
        info = capi.QkTopoInfo()

        def surgery():
            capi.check(capi.lib().qk_update_topology(
                ctypes.byref(base.t), ctypes.byref(nt), ctypes.byref(e), 0, bins,
                ctypes.byref(info), ws.data_ptr(), nb, capi._stream()), "qk_update_topology")

        s_ms = timed_ms(surgery)
        fresh = capi.DeviceTree(kind, new_d, builder=builder, sah_bins=bins)
        b_ms = timed_ms(fresh.build)
        entry = {"edited": int(len(dele) + len(ins) + app + len(mov)), "surgery_ms": round(s_ms, 4),
                 "rebuild_ms": round(b_ms, 4), "ratio": round(s_ms / b_ms, 3),
                 "rebuilt_subtrees": info.cuts, "rebuilt_leaves": info.new_leaves,
                 "spliced": info.spliced, "fallback": bool(info.rebuild)}
        if not info.rebuild:
            base.update_topology(new_d, dele, ins, mov)
            same = (torch.equal(base.closest(queries_d), fresh.closest(queries_d)) and
                    torch.equal(base.knn(queries_d, 8), fresh.knn(queries_d, 8)))
            if rays_d is not None:
                same = same and torch.equal(base.raycast(rays_d), fresh.raycast(rays_d))
            if not same:
                raise RuntimeError(f"topology {mode}: edited tree answers differently")
            entry["depth"] = base.depth
            entry["fresh_depth"] = fresh.depth
        if mode == "cluster":
            entry["api"] = topology_api_wall(kind, items, new, dele, ins, mov, builder)
        out[f"{mode}_1pct"] = entry
        del base, fresh, arrays, ws
    return out


def topology_api_wall(kind, items, new, dele, ins, mov, builder, rounds=4):
    """Host wall time through the module (the C++ updateBVHGPU: it uploads only the edit
    script and the primitives it brings, and reuses its arrays from the previous edit) in
    steady state -- one object takes `rounds` further 1% edits of the same kind after the first
    (which allocates), the later ones timed -- against constructing the object from the whole
    edited scene (conversion, allocation, upload, build).  Medians."""
    import time

    import torch

    import quarry
    from quarry import workloads as w

    wrap = (lambda a: a.reshape(-1, 3, 3)) if kind == "tri" else (lambda a: a)
    make = {"tri": lambda a: quarry.Scene(wrap(a), builder=builder),
            "point": lambda a: quarry.PointCloud(a, builder=builder)}[kind]
    obj = make(items)
    obj.update_topology(wrap(new), deleted=dele, moved=mov, inserted=ins)
    cur = new
    upd, reb, inner, full = [], [], [], 0
    for r in range(rounds):
        nxt, d2, i2, m2 = w.topology_edit(cur, 0.01, "cluster", 100 + r)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tm = obj.update_topology(wrap(nxt), deleted=d2, moved=m2, inserted=i2)
        upd.append((time.perf_counter() - t0) * 1e3)
        inner.append(float(tm["total_ms"]))
        full += int(bool(tm["full_rebuild"]))
        t0 = time.perf_counter()
        fresh = make(nxt)
        reb.append((time.perf_counter() - t0) * 1e3)
        del fresh
        cur = nxt
    u, r = float(np.median(upd[1:])), float(np.median(reb[1:]))
    return {"update_wall_ms": round(u, 3), "rebuild_wall_ms": round(r, 3), "ratio": round(u / r, 3),
            "update_cpp_total_ms": round(float(np.median(inner[1:])), 3),
            "full_rebuilds": full, "rounds": rounds, "timed": "rounds 2..n, cluster 1% each",
            "note": "walls include the module's host conversion of the whole scene (both paths)"}


# ---------------------------------------------------------------------------------------
# point clouds: closest / kNN8 / radius 1.0 and the 1% coherent refit
# ---------------------------------------------------------------------------------------
def points_arm(args, world, rank, local):
    """1,048,576 points on a noisy sphere (r=50, radial N(0,0.5)) and 1,048,576 uniform in
    [0,100]^3; per cloud 20,000 queries uniform in its bounds for closest, kNN (k=8) and
    radius (r=1.0).  A step answers all six query sets (L2 flushed before each step).  The
    refit moves a spatially coherent 1% of the points by N(0, 0.05) per axis."""
    import torch

    import oracle
    from quarry import capi, workloads as w

    torch.cuda.set_device(local)
    n = 65_536 if args.small else 1_048_576
    nq, k, r = 20_000, 8, 1.0
    seed = 1 + rank
    l2 = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    clouds = {}
    for kind in ("surface", "volume"):
        pts = w.point_cloud(kind, n, seed)
        lo, hi = pts.min(axis=0), pts.max(axis=0)
        q = w.uniform_points(nq, lo, hi, seed, 13)
        trees = {}
        for bname, builder, bins in (("lbvh", "lbvh", 32), ("sah8", "sah", 8), ("sah32", "sah", 32)):
            trees[bname] = capi.DeviceTree("point", pts, builder=builder, sah_bins=bins)
            trees[bname].build_wide()
        clouds[kind] = {"pts": pts, "q": q, "q_d": capi.to_device(q, np.float32),
                        "tree": trees["lbvh"], "trees": trees}
        if args.dump and rank == 0:
            from quarry import dumps

            Path(args.dump).mkdir(parents=True, exist_ok=True)
            dumps.write_qrcd(Path(args.dump) / f"points_{kind}.qrcd", pts, q)

    def timed(fn, steps, warm=3):
        for _ in range(warm):
            fn()
        ts = []
        for _ in range(steps):
            l2.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return ts

    outs = {}
    ops = ("closest", "knn", "radius")

    def run(kind, op, tree, flags):
        c = clouds[kind]
        if op == "closest":
            outs[(kind, op)] = tree.closest(c["q_d"], flags)
        elif op == "knn":
            outs[(kind, op)] = tree.knn(c["q_d"], k, flags)
        else:
            outs[(kind, op)] = tree.radius(c["q_d"], r, flags)

    def snapshot(key):
        v = outs[key]
        return (v[0].cpu().numpy(), v[1].cpu().numpy()) if isinstance(v, tuple) else v.cpu().numpy()

    def same(a, b):
        return (np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
                if isinstance(a, tuple) else np.array_equal(a, b))

    # Every (cloud, operation) takes its fastest (tree, schedule): the sphere shell's queries
    # have a heavy tail that the warp-per-query kernels spread out, the uniform cloud's do not.
    # All candidates must return the bits of the LBVH thread-per-query run.
    variants = {"bin": 0, "bin_morton": capi.QK_ORDER_MORTON, "wide": capi.QK_WIDE,
                "wide_morton": capi.QK_WIDE | capi.QK_ORDER_MORTON,
                "split": capi.QK_TUNE_SPLIT, "split_morton": capi.QK_TUNE_SPLIT | capi.QK_ORDER_MORTON,
                "leaf4": capi.QK_TUNE_LEAF4, "leaf4_morton": capi.QK_TUNE_LEAF4 | capi.QK_ORDER_MORTON,
                "bin_coh": capi.QK_ORDER_COHERENT, "split_coh": capi.QK_TUNE_SPLIT | capi.QK_ORDER_COHERENT,
                "leaf4_coh": capi.QK_TUNE_LEAF4 | capi.QK_ORDER_COHERENT}
    radius_variants = {"stash": capi.QK_TUNE_STASH,
                       "stash_morton": capi.QK_TUNE_STASH | capi.QK_ORDER_MORTON,
                       "stash_leaf4": capi.QK_TUNE_STASH | capi.QK_TUNE_LEAF4,
                       "stash_coh": capi.QK_TUNE_STASH | capi.QK_ORDER_COHERENT}
    vms, plan = {}, {}
    for kind, c in clouds.items():
        for op in ops:
            run(kind, op, c["trees"]["lbvh"], 0)
            base = snapshot((kind, op))
            cands = {**variants, **radius_variants} if op == "radius" else variants
            for bname, tree in c["trees"].items():
                for vname, f in cands.items():
                    run(kind, op, tree, f)
                    if not same(base, snapshot((kind, op))):
                        raise RuntimeError(f"{kind} {op}: {bname}/{vname} differs")
                    t = float(np.median(timed(lambda: run(kind, op, tree, f), 5)))
                    vms[f"{kind}/{op}/{bname}/{vname}"] = t
                    if (kind, op) not in plan or t < plan[(kind, op)][2]:
                        plan[(kind, op)] = (bname, vname, t)

    variants.update(radius_variants)

    def step():
        for (kind, op), (bname, vname, _) in plan.items():
            run(kind, op, clouds[kind]["trees"][bname], variants[vname])

    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ts = timed(step, args.steps, args.warmup)
    clocks = clk.summary()
    ms = max_over_ranks(world, float(np.mean(ts)))
    queries = 2 * 3 * nq
    value = world * queries / (ms * 1e-3) / 1e6

    # per-operation kernel times and the canonical visit counts (binary LBVH) for the roofline
    per_op = {}
    for op in ops:
        def one(op=op):
            for kind in clouds:
                bname, vname, _ = plan[(kind, op)]
                run(kind, op, clouds[kind]["trees"][bname], variants[vname])
        per_op[op] = float(np.median(timed(one, 20)))
    stats = torch.zeros(4, dtype=torch.int64, device="cuda")
    for c in clouds.values():
        c["tree"].knn(c["q_d"], k, 0, stats=stats)
    st = stats.cpu().numpy()
    p_leaf = st[1] / (2 * nq)
    p_int = (st[0] - st[1]) / (2 * nq)
    bytes_per_q = 12 + 8 * k + 96 * p_int + (32 + 12 + 4) * p_leaf
    pk, pk_kind = peaks()
    achieved = bytes_per_q * 2 * nq / (per_op["knn"] * 1e-3) / 1e9

    def kernel_of(op, vname):
        f = variants[vname]
        return ("k_%s_wide" if f & capi.QK_WIDE else "k_%s_split" if f & capi.QK_TUNE_SPLIT
                else "k_%s_bin") % op

    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4), "traffic": None,
                "peak_kind": pk_kind,
                "kernel": ", ".join(f"{kernel_of('knn', plan[(kind, 'knn')][1])} ({kind})"
                                    for kind in clouds),
                "kernel_ms": round(per_op["knn"], 4), "bytes_per_query": round(float(bytes_per_q), 1),
                "canonical_counts": {"internal_pops_per_query": round(float(p_int), 2),
                                     "leaf_tests_per_query": round(float(p_leaf), 2)}}

    # ---- refit: 1% coherent motion, dirty refit vs full refit vs rebuild ----
    refit = {}
    for kind, c in clouds.items():
        moved, ids = w.coherent_motion(c["pts"], 0.01, 0.05, seed)
        t = c["tree"]
        ids_d = capi.to_device(ids, np.int32)
        sub_moved = capi.to_device(moved[ids], np.float32)
        sub_orig = capi.to_device(c["pts"][ids], np.float32)
        flip = [0]

        def dirty():
            t.refit_dirty(ids_d, sub_moved if flip[0] % 2 == 0 else sub_orig)
            flip[0] += 1

        d_ms = float(np.median(timed(dirty, 10, 2)))
        if flip[0] % 2 == 1:  # leave the tree on the moved points
            pass
        else:
            t.refit_dirty(ids_d, sub_moved)
        moved_d = capi.to_device(moved, np.float32)
        f_ms = float(np.median(timed(lambda: t.refit(moved_d), 10, 2)))
        fresh = capi.DeviceTree("point", moved_d)
        b_ms = float(np.median(timed(lambda: fresh.build(), 5, 1)))
        fresh.build_wide()
        a = t.knn(c["q_d"], k, 0).cpu().numpy()
        b = fresh.knn(c["q_d"], k, 0).cpu().numpy()
        ref = oracle.LBVH("point", moved)
        want = ref.knn(c["q"], k)
        if not (np.array_equal(a.view(np.uint32), want) and np.array_equal(b.view(np.uint32), want)):
            raise RuntimeError(f"{kind}: refit kNN differs from the rebuild or the oracle")
        ca = t.closest(c["q_d"], 0).cpu().numpy().view(np.uint32)
        if not np.array_equal(ca, ref.closest(c["q"])):
            raise RuntimeError(f"{kind}: refit closest differs from the oracle")
        refit[kind] = {"dirty": int(ids.size), "dirty_refit_ms": round(d_ms, 4),
                       "full_refit_ms": round(f_ms, 4), "rebuild_ms": round(b_ms, 4),
                       "knn_fingerprint_after_refit": f"0x{oracle.knn_hash(want):016x}"}
        t.refit(capi.to_device(c["pts"], np.float32))

    # ---- topology edits (1%, cluster / scatter) on the surface cloud's LBVH ----
    topology = topology_timing("point", clouds["surface"]["pts"], "lbvh", 32,
                               clouds["surface"]["q_d"], seed,
                               lambda fn: float(np.median(timed(fn, 5, 2))))

    # ---- end to end: queries from pinned host memory, results read back ----
    host_q = {kind: torch.from_numpy(c["q"]).pin_memory() for kind, c in clouds.items()}

    def e2e():
        total = 0
        for kind, c in clouds.items():
            qd = host_q[kind].to("cuda", non_blocking=True)
            tc, fc = c["trees"][plan[(kind, "closest")][0]], variants[plan[(kind, "closest")][1]]
            tk, fk = c["trees"][plan[(kind, "knn")][0]], variants[plan[(kind, "knn")][1]]
            tr, fr = c["trees"][plan[(kind, "radius")][0]], variants[plan[(kind, "radius")][1]]
            a = tc.closest(qd, fc)
            b = tk.knn(qd, k, fk)
            off, keys = tr.radius(qd, r, fr)
            a.cpu(), b.cpu(), off.cpu(), keys.cpu()
            total += int(keys.numel())
        return total

    et = timed(e2e, 10)
    e2e_ms = max_over_ranks(world, float(np.mean(et)))
    radius_keys = sum(int(outs[(kind, "radius")][1].numel()) for kind in clouds)

    line = None
    if rank == 0:
        # quarry's CPU reference on the same queries, all host threads
        threads = os.cpu_count() or 1
        parity, cpu_ms, kind_ref = {}, 0.0, "port"
        if oracle.REF_PATH.exists():
            R = oracle.Reference()
            kind_ref = "reference"
            for kind, c in clouds.items():
                cw, cms, _ = R.closest("point", c["pts"], c["q"], threads)
                kw_, kms, _ = R.knn("point", c["pts"], c["q"], k, threads)
                ro, rk, rms = R.radius("point", c["pts"], c["q"], r, threads)
                cpu_ms += cms + kms + rms
                ok = (np.array_equal(outs[(kind, "closest")].cpu().numpy().view(np.uint32), cw)
                      and np.array_equal(outs[(kind, "knn")].cpu().numpy().view(np.uint32), kw_)
                      and np.array_equal(outs[(kind, "radius")][0].cpu().numpy(), ro)
                      and np.array_equal(outs[(kind, "radius")][1].cpu().numpy().view(np.uint64), rk))
                if not ok:
                    raise RuntimeError(f"{kind}: results differ from the CPU reference")
                parity[kind] = {"closest": f"0x{oracle.closest_hash(cw):016x}",
                                "knn": f"0x{oracle.knn_hash(kw_):016x}",
                                "radius": f"0x{oracle.radius_hash(ro, rk):016x}"}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mqueries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generators, identical bytes on every host)",
            "config": {"workload": "points", "points_per_cloud": n, "clouds": ["surface", "volume"],
                       "queries_per_op": nq, "k": k, "radius": r,
                       "plan": {f"{kind}/{op}": f"{b}/{v}" for (kind, op), (b, v, _) in plan.items()},
                       "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": f"replica x{world}"},
            "variants_ms": {kk: round(v, 4) for kk, v in vms.items()},
            "per_op_ms": {kk: round(v, 4) for kk, v in per_op.items()},
            "radius_results": radius_keys, "refit": refit, "topology": topology,
            "parity": {"against": kind_ref, "fingerprints": parity,
                       "variants": "all trees / layouts / orders / schedules bit-identical"},
            "roofline": roofline,
            "cpu_baseline": {"value": round(queries / (cpu_ms * 1e-3) / 1e6, 4) if cpu_ms else None,
                             "unit": "Mqueries/s", "cores": threads, "kind": kind_ref,
                             "sample": "all 120,000 queries of the step; CPU tree builds excluded"},
            "clocks": clocks,
            "e2e": {"value": round(world * queries / (e2e_ms * 1e-3) / 1e6, 2),
                    "unit": "Mqueries/s", "h2d_bytes_per_step": 2 * nq * 12,
                    "d2h_bytes_per_step": 2 * nq * (8 + 8 * k + 4) + 8 * radius_keys,
                    "path": "pinned queries -> qk_closest / qk_knn / qk_radius_count+fill -> host"},
            "gpu_launches": None,
        }
        # per cloud: closest, kNN (1 + order each), radius count (1 + scan 3 + order) + fill
        # (1 + order) + 4 segment-sort launches; a Morton order is 24 launches, a coherent
        # order 4 (grid, keys, scan, scatter)
        launches = 0
        for (kind, op), (_, vname, _) in plan.items():
            morton = (24 if variants[vname] & capi.QK_ORDER_MORTON else
                      4 if variants[vname] & capi.QK_ORDER_COHERENT else 0)
            launches += (1 + morton) if op != "radius" else (4 + morton) + (1 + morton) + 4
        line["gpu_launches"] = args.steps * launches
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# batched uneven scenes: one CUDA graph per step vs the per-scene launch loop
# ---------------------------------------------------------------------------------------
def batch_arm(args, world, rank, local):
    """256 scenes (128 terrains of 1k..500k triangles, 128 uniform clouds of 4k..1M points,
    1k..100k queries each: closest / kNN16 / radius at 0.02 x diagonal, plus as many rays on
    the terrains).  A step builds every tree and answers every query.  Batched: one CUDA graph
    of one-launch-per-phase kernels (launch shapes from the autotuner).  Loop: the same work
    through the single-tree calls, scene after scene.  Each rank runs its own 256 scenes."""
    import torch

    import oracle
    from quarry import autotune, pipeline, workloads as w

    torch.cuda.set_device(local)
    kw = {}
    if args.small:
        kw = dict(terrains=16, clouds=16, tri_range=(1_000, 50_000),
                  point_range=(4_000, 100_000), query_range=(1_000, 10_000))
    t0 = time.perf_counter()
    cfg = w.batch_config(first_seed=1000 + 100_000 * rank, **kw)
    gen_s = time.perf_counter() - t0
    pipe = pipeline.BatchPipeline(cfg.terrains, cfg.clouds, cfg.k)
    pipe.size_radius_outputs()
    tuner = autotune.Autotuner(args.tune_cache)
    tune_report = pipe.tune(tuner, force=args.retune)
    pipe.size_radius_outputs()
    tune_report["builder"] = pipe.tune_builder(tuner, force=args.retune)
    pipe.capture()
    for _ in range(max(args.warmup, 3)):
        pipe.replay()
    torch.cuda.synchronize()
    pipe.sync()

    # ---- batched: K graph replays (inputs are GBs, larger than L2) ----
    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with Clocks(local) as clk:
        for e0, e1 in ev:
            e0.record()
            pipe.replay()
            e1.record()
        torch.cuda.synchronize()
    clocks = clk.summary()
    batched_ms = max_over_ranks(world, float(np.mean([a.elapsed_time(b) for a, b in ev])))
    pipe.sync()
    got = pipe.results()

    # ---- the per-scene launch loop, same layouts and orders ----
    loop_steps = 2 if args.small else 3
    pipe.run_loop()
    torch.cuda.synchronize()
    lt = []
    for _ in range(loop_steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pipe.run_loop()
        e1.record()
        torch.cuda.synchronize()
        lt.append(e0.elapsed_time(e1))
    loop_ms = max_over_ranks(world, float(np.mean(lt)))
    loop = pipe.results(loop_layout=True)
    mism = []
    for key, per in got.items():
        for i, (a, b) in enumerate(zip(per, loop[key])):
            same = (np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
                    if isinstance(a, tuple) else np.array_equal(a, b))
            if not same:
                mism.append(f"{key}[{i}]")
    if mism:
        raise RuntimeError(f"batched and loop results differ: {mism[:8]}")

    # ---- end to end: inputs uploaded from pinned host memory, results read back ----
    host_in = [(t, torch.empty(t.shape, dtype=t.dtype).pin_memory().copy_(t.cpu()))
               for t in [b.items for b in pipe.batches.values()] + [ph.inputs for ph in pipe.phases]]
    outs = []
    for ph in pipe.phases:
        outs.append((ph.out, torch.empty(ph.out.shape, dtype=ph.out.dtype).pin_memory()))
        if ph.offsets is not None:
            outs.append((ph.offsets, torch.empty(ph.offsets.shape, dtype=ph.offsets.dtype).pin_memory()))
    h2d = int(sum(h.numel() * h.element_size() for _, h in host_in))
    d2h = int(sum(h.numel() * h.element_size() for _, h in outs))

    def e2e_step():
        for d, h in host_in:
            d.copy_(h, non_blocking=True)
        pipe.replay()
        for d, h in outs:
            h.copy_(d, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    et = []
    for _ in range(min(args.steps, 5)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        e2e_step()
        e1.record()
        torch.cuda.synchronize()
        et.append(e0.elapsed_time(e1))
    e2e_ms = max_over_ranks(world, float(np.mean(et)))
    nq = pipe.query_count()

    line = None
    if rank == 0:
        # ---- quarry's CPU reference on sample scenes: smallest, median and largest of each kind
        threads = os.cpu_count() or 1
        checked, cpu_q, cpu_ms = [], 0, 0.0
        have_ref = oracle.REF_PATH.exists()
        R = oracle.Reference() if have_ref else None
        sample_sets = () if args.no_cpu_baseline else (("tri", cfg.terrains), ("point", cfg.clouds))
        for kind, scenes in sample_sets:
            order = np.argsort([s.items.shape[0] for s in scenes], kind="stable")
            for i in sorted({int(order[0]), int(order[len(order) // 2]), int(order[-1])}):
                sc = scenes[i]
                if R is not None:
                    want = {"closest": R.closest(kind, sc.items, sc.closest, threads),
                            "knn": R.knn(kind, sc.items, sc.knn, cfg.k, threads),
                            "radius": R.radius(kind, sc.items, sc.radius, float(sc.r), threads)}
                    if kind == "tri":
                        want["rays"] = R.raycast(sc.items, sc.rays, threads)
                    for name, wv in want.items():
                        cpu_ms += wv[-2] if name != "radius" else wv[-1]
                    res = {k: (v[0] if k != "radius" else (v[0], v[1])) for k, v in want.items()}
                else:
                    ref = oracle.LBVH(kind, sc.items)
                    ta = time.perf_counter()
                    res = {"closest": ref.closest(sc.closest, threads),
                           "knn": ref.knn(sc.knn, cfg.k, threads),
                           "radius": ref.radius(sc.radius, float(sc.r), threads)}
                    if kind == "tri":
                        res["rays"] = ref.raycast(sc.rays, threads)
                    cpu_ms += (time.perf_counter() - ta) * 1e3
                for name, wv in res.items():
                    g = got[f"{kind}_{name}"][i]
                    ok = (np.array_equal(g[0], wv[0]) and np.array_equal(g[1], wv[1])
                          if name == "radius" else np.array_equal(g, wv))
                    if not ok:
                        raise RuntimeError(f"{kind} scene {i} {name} differs from the CPU reference")
                    cpu_q += len(g[0]) - 1 if name == "radius" else len(g)
                checked.append(f"{kind}[{i}] n={sc.items.shape[0]}")
        speedup = loop_ms / batched_ms
        line = {
            "metric": METRIC, "value": round(speedup, 3), "unit": "x (per-scene loop / batched)",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": round(batched_ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generators, identical bytes on every host)",
            "config": {"workload": "batch", "scenes": len(cfg.terrains) + len(cfg.clouds),
                       "terrains": len(cfg.terrains), "clouds": len(cfg.clouds),
                       "triangles": int(sum(s.items.shape[0] for s in cfg.terrains)),
                       "points": int(sum(s.items.shape[0] for s in cfg.clouds)),
                       "queries": nq, "k": cfg.k,
                       "l2": "inputs and trees (GBs) larger than L2; no flush",
                       "parallelism": f"{world} rank(s), each its own 256 scenes",
                       "builder": pipe.builder,
                       "step": "build every tree + every query of every scene"},
            "batched": {"ms": round(batched_ms, 3),
                        "mqueries_per_s": round(world * nq / (batched_ms * 1e-3) / 1e6, 2),
                        "graph_kernel_nodes": pipe.graph_kernel_nodes()},
            "loop": {"ms": round(loop_ms, 3), "steps": loop_steps,
                     "mqueries_per_s": round(world * nq / (loop_ms * 1e-3) / 1e6, 2)},
            "autotune": tune_report, "tune_cache": str(tuner.path),
            "parity": {"batched_vs_loop": "all scenes bit-identical",
                       "cpu_reference_scenes": checked,
                       "against": "reference" if have_ref else "port"},
            "roofline": None,
            "cpu_baseline": {"value": round(cpu_q / (cpu_ms * 1e-3) / 1e6, 4) if cpu_ms else None,
                             "unit": "Mqueries/s", "cores": threads,
                             "kind": "reference" if have_ref else "port",
                             "sample": "queries of the smallest, median and largest scene of "
                                       "each kind; CPU tree builds excluded"},
            "clocks": clocks,
            "e2e": {"value": round(world * nq / (e2e_ms * 1e-3) / 1e6, 2), "unit": "Mqueries/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "path": "pinned host inputs -> graph replay -> pinned host outputs"},
            "generate_s": round(gen_s, 1),
            "gpu_launches": (pipe.graph_kernel_nodes() or 0) * args.steps,
        }
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------
def main():
    args = parse()
    world, rank, local = init_dist(args)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        elif args.workload == "grad":
            grad_arm(args, world, rank, local)
        elif args.workload == "batch":
            batch_arm(args, world, rank, local)
        elif args.workload == "points":
            points_arm(args, world, rank, local)
        else:
            rays_arm(args, world, rank, local)
        barrier(world)
    finally:
        from quarry import dist

        if _RANKS is not None:
            dist.destroy(_RANKS)


def rays_arm(args, world, rank, local):
    """City (default) or terrain: rays through the engine, the timed step."""
    import torch

    import oracle
    from quarry import capi

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfg, desc = make_workload(args.workload, args.small, rank)
    nrays = cfg.rays.shape[0]
    if args.dump and rank == 0:
        from quarry import dumps

        Path(args.dump).mkdir(parents=True, exist_ok=True)
        dumps.write_qryd(Path(args.dump) / f"{args.workload}.qryd", cfg.tris, cfg.queries)

    # ---- builds (timed beside the step): LBVH and binned SAH with 32 bins ----
    tris_d = capi.to_device(cfg.tris, np.float32)

    def timed_build(builder):
        """Device build time (CUDA events) of qk_build from device-resident triangles; the
        call includes its depth read-back (and the SAH level read-backs)."""
        tr = capi.DeviceTree("tri", tris_d, builder=builder, sah_bins=32)
        times = []
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            tr.build()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        tr.build_wide()
        return tr, float(np.median(times))

    trees, build_ms = {}, {}
    for b in ("lbvh", "sah"):
        trees[b], build_ms[b] = timed_build(b)

    rays_d = capi.to_device(cfg.rays, np.float32)
    q_d = capi.to_device(cfg.queries, np.float32)
    l2_flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    dyn, occ, mort = capi.QK_TUNE_DYNAMIC, capi.QK_TUNE_HIGH_OCC, capi.QK_ORDER_MORTON
    coh = capi.QK_ORDER_COHERENT
    modes = {"bin": 0, "bin_morton": mort, "wide": capi.QK_WIDE,
             "wide_morton": capi.QK_WIDE | mort, "bin_occ": occ, "bin_morton_occ": mort | occ,
             "bin_dyn": dyn, "bin_morton_dyn": mort | dyn, "bin_morton_dyn_occ": mort | dyn | occ,
             "bin_sm": capi.QK_TUNE_SHORT_STACK, "bin_occ_sm": occ | capi.QK_TUNE_SHORT_STACK,
             "bin_leaf4": capi.QK_TUNE_LEAF4, "bin_occ_leaf4": occ | capi.QK_TUNE_LEAF4,
             "bin_morton_occ_leaf4": mort | occ | capi.QK_TUNE_LEAF4,
             "bin_coh": coh, "bin_coh_occ": coh | occ, "bin_coh_dyn_occ": coh | dyn | occ,
             "bin_coh_occ_leaf4": coh | occ | capi.QK_TUNE_LEAF4, "wide_coh": capi.QK_WIDE | coh}
    variants = {f"{b}_{m}": (b, f) for b in trees for m, f in modes.items()}
    if args.only:
        variants = {args.only: variants[args.only]}

    base = trees["lbvh"].raycast(rays_d, 0).clone()
    # every variant must give the same bits
    for name, (b, flags) in variants.items():
        got = trees[b].raycast(rays_d, flags)
        if not torch.equal(got, base):
            raise RuntimeError(f"variant {name} differs from the LBVH binary results")

    def time_variant(tree, flags, steps, warmup):
        out = torch.empty(nrays, dtype=torch.int64, device=dev)
        ws = torch.empty(capi.lib().qk_query_workspace_bytes(nrays, flags), dtype=torch.uint8,
                         device=dev)
        for _ in range(warmup):
            tree.raycast(rays_d, flags, out=out, ws=ws)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for e0, e1 in ev:
            l2_flush.zero_()
            e0.record()
            tree.raycast(rays_d, flags, out=out, ws=ws)
            e1.record()
        torch.cuda.synchronize()
        return [e0.elapsed_time(e1) for e0, e1 in ev]

    results = {}
    for name, (b, flags) in variants.items():
        results[name] = float(np.median(time_variant(trees[b], flags, 10, 3)))
    best = min(results, key=results.get)
    best_builder, best_flags = variants[best]
    tree = trees[best_builder]

    # canonical per-ray visit counts: binary traversal of the timed tree (roofline bytes)
    stats = torch.zeros(4, dtype=torch.int64, device=dev)
    tree.raycast(rays_d, 0, stats=stats)
    s = stats.cpu().numpy()
    node_tests, tri_tests, overflows = int(s[0]), int(s[1]), int(s[2])
    if overflows:
        raise RuntimeError(f"{overflows} rays overflowed the traversal stack")
    p_int = (node_tests - tri_tests) / nrays
    p_leaf = tri_tests / nrays
    bytes_per_ray = 40.0 + 96.0 * p_int + (32.0 + 36.0) * p_leaf

    # ---- the timed steps of the headline variant ----
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        step_ms = time_variant(tree, best_flags, args.steps, args.warmup)
    clocks = clk.summary()
    ms = float(np.sum(step_ms)) / args.steps
    ms = max_over_ranks(world, ms)
    value = world * nrays / (ms * 1e-3) / 1e6

    # ---- roofline: traversal kernel alone on pre-sorted rays ----
    # the engine's coherent or Morton order (quantize10 of src/gpu/morton.h), recomputed on
    # the host, so the kernel alone can be timed on rays that are already in that order
    trav_flags = best_flags & ~(capi.QK_ORDER_MORTON | capi.QK_ORDER_COHERENT)
    if best_flags & capi.QK_ORDER_COHERENT:
        sorted_rays = capi.to_device(cfg.rays[coherent_order(cfg.rays)], np.float32)
    elif best_flags & capi.QK_ORDER_MORTON:
        o = cfg.rays[:, :3]
        lo, hi = o.min(0), o.max(0)
        qz = np.clip((o - lo) / np.where(hi > lo, hi - lo, 1), 0, 1)
        qi = (qz * 1023 + 0.5).astype(np.uint32)

        def spread(v):
            v = v & 0x3FF
            v = (v | (v << 16)) & 0x030000FF
            v = (v | (v << 8)) & 0x0300F00F
            v = (v | (v << 4)) & 0x030C30C3
            v = (v | (v << 2)) & 0x09249249
            return v

        code = spread(qi[:, 0]) | (spread(qi[:, 1]) << 1) | (spread(qi[:, 2]) << 2)
        order = np.argsort(code, kind="stable")
        sorted_rays = capi.to_device(cfg.rays[order], np.float32)
    else:
        sorted_rays = rays_d
    out = torch.empty(nrays, dtype=torch.int64, device=dev)
    ws = torch.empty(capi.lib().qk_query_workspace_bytes(nrays, trav_flags), dtype=torch.uint8,
                     device=dev)
    for _ in range(3):
        tree.raycast(sorted_rays, trav_flags, out=out, ws=ws)
    kt = []
    for _ in range(20):
        l2_flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tree.raycast(sorted_rays, trav_flags, out=out, ws=ws)
        e1.record()
        torch.cuda.synchronize()
        kt.append(e0.elapsed_time(e1))
    kernel_ms = float(np.median(kt))
    pk, pk_kind = peaks()
    achieved = bytes_per_ray * nrays / (kernel_ms * 1e-3) / 1e9
    traffic = profiled_traffic(args.workload, best)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4),
                "traffic": traffic, "peak_kind": pk_kind,
                "kernel": ("k_ray_wide" if trav_flags & capi.QK_WIDE else
                           "k_ray_bin_dyn" if trav_flags & capi.QK_TUNE_DYNAMIC else "k_ray_bin"),
                "tree": best_builder,
                "kernel_ms": round(kernel_ms, 4),
                "kernel_timing": ("the traversal alone, CUDA events, on rays already in the "
                                  "variant's order (contiguous)"),
                # the same bytes over the whole timed step (ordering kernels included)
                "frac_step": round(bytes_per_ray * nrays / (ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4),
                "bytes_per_ray": round(bytes_per_ray, 1),
                "canonical_counts": {"node_tests_per_ray": round(node_tests / nrays, 3),
                                     "tri_tests_per_ray": round(p_leaf, 3)}}

    # ---- kNN and build beside the step ----
    k_out = torch.empty((q_d.shape[0], 8, 2), dtype=torch.int32, device=dev)
    knn_base = tree.knn(q_d, 8, 0).clone()
    knn_ms_by = {}
    for kname, kf in (("layout_of_rays", best_flags & (capi.QK_WIDE | capi.QK_ORDER_MORTON |
                                                       capi.QK_ORDER_COHERENT)),
                      ("input", 0),
                      ("split", capi.QK_TUNE_SPLIT),
                      ("split_morton", capi.QK_TUNE_SPLIT | capi.QK_ORDER_MORTON),
                      ("split_coherent", capi.QK_TUNE_SPLIT | capi.QK_ORDER_COHERENT),
                      ("leaf4", capi.QK_TUNE_LEAF4),
                      ("leaf4_morton", capi.QK_TUNE_LEAF4 | capi.QK_ORDER_MORTON)):
        for _ in range(3):
            tree.knn(q_d, 8, kf, out=k_out)
        if not torch.equal(k_out, knn_base):
            raise RuntimeError(f"kNN variant {kname} differs")
        kt = []
        for _ in range(10):
            l2_flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            tree.knn(q_d, 8, kf, out=k_out)
            e1.record()
            torch.cuda.synchronize()
            kt.append(e0.elapsed_time(e1))
        knn_ms_by[kname] = float(np.median(kt))
    knn_variant = min(knn_ms_by, key=knn_ms_by.get)
    knn_ms = knn_ms_by[knn_variant]

    # ---- topology edits on the SAH tree (the surgery path; results checked at full size) ----
    def med_ms(fn, steps=5):
        for _ in range(2):
            fn()
        ts = []
        for _ in range(steps):
            l2_flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    topology = None
    if args.workload == "city":
        topology = topology_timing("tri", cfg.tris, "sah", 32, q_d, 1 + rank, med_ms,
                                   rays_d[:200_000])

    # ---- e2e through the C ABI from pinned host buffers: qk_raycast_host uploads, traces and
    # reads back in chunks (uploads, traversals and read-backs on three streams), all inside
    # the timed region ----
    host_rays = torch.from_numpy(np.ascontiguousarray(cfg.rays)).pin_memory()
    host_out = torch.empty(nrays, dtype=torch.int64).pin_memory()
    dev_rays = torch.empty((nrays, 8), dtype=torch.float32, device=dev)
    streams = tuple(torch.cuda.Stream() for _ in range(4))

    def e2e_call(chunks, flags, ws):
        if chunks == 0:
            # zero-copy: the traversal reads the pinned rays and writes the pinned results
            with torch.cuda.stream(streams[0]):
                tree.raycast_mapped(host_rays, host_out, flags, ws)
        elif chunks < 0:
            # copy pipeline for the rays; the traversals store results into pinned host_out
            tree.raycast_host(host_rays, host_out, dev_rays, None, flags, -chunks, streams, ws)
        else:
            tree.raycast_host(host_rays, host_out, dev_rays, out, flags, chunks, streams, ws)

    def e2e_times(chunks, steps, flags):
        nb = (capi.lib().qk_query_workspace_bytes(nrays, flags) if chunks == 0 else
              capi.lib().qk_raycast_host_workspace_bytes(nrays, abs(chunks)))
        ws = torch.empty(nb, dtype=torch.uint8, device=dev)
        for _ in range(3):
            e2e_call(chunks, flags, ws)
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            l2_flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(streams[0])
            for x in streams[1:]:
                x.wait_event(e0)
            e2e_call(chunks, flags, ws)
            ends = [torch.cuda.Event(enable_timing=True) for _ in streams]
            for ev, x in zip(ends, streams):
                ev.record(x)
            torch.cuda.synchronize()
            ts.append(max(e0.elapsed_time(ev) for ev in ends))
        return ts

    # the transfer scheme (copy pipeline with 2-16 chunks, or zero-copy through mapped pinned
    # memory) and the ray order are chosen by measurement (same bits for every choice): per
    # chunk, an order costs a fixed few tens of microseconds
    orders = {"timed variant": best_flags,
              "input order": best_flags & ~(capi.QK_ORDER_MORTON | capi.QK_ORDER_COHERENT)}
    schemes = {"zero-copy": 0, **{f"{c} chunks": c for c in (2, 4, 8, 16)},
               **{f"{c} chunks, results stored to host": -c for c in (4, 8, 16)}}
    chunk_ms = {f"{sc}, {o}": float(np.median(e2e_times(c, 10, f)))
                for o, f in orders.items() for sc, c in schemes.items()}
    e2e_pick = min(chunk_ms, key=chunk_ms.get)
    scheme, order_name = e2e_pick.rsplit(", ", 1)
    chunks = schemes[scheme]
    e2e_flags = orders[order_name]
    e2e_t = e2e_times(chunks, min(args.steps, 50), e2e_flags)
    if not np.array_equal(host_out.numpy(), tree.raycast(rays_d, 0).cpu().numpy()):
        raise RuntimeError("e2e results differ from the device-resident run")
    e2e_ms = max_over_ranks(world, float(np.mean(e2e_t)))
    e2e_value = world * nrays / (e2e_ms * 1e-3) / 1e6

    result = host_out.numpy().view(np.uint64)
    fp, hits = oracle.ray_hash(result)

    line = None
    if rank == 0:
        cpu = None
        parity = None
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            sample = min(nrays, 200_000 if not args.small else 50_000)
            ref_out, ref_ms, ref_build, kind = cpu_reference_rays(cfg.tris, cfg.rays[:sample],
                                                                  threads)
            mism = int((ref_out != result[:sample]).sum())
            parity = {"checked_rays": sample, "mismatches": mism, "against": kind}
            if mism:
                raise RuntimeError(f"{mism} of {sample} rays differ from the CPU reference")
            cpu = {"value": round(sample / (ref_ms * 1e-3) / 1e6, 4), "unit": "Mrays/s",
                   "cores": threads, "kind": kind,
                   "sample": f"first {sample} of the {nrays} rays, reference BVH build "
                             f"({ref_build:.0f} ms) excluded"}
            # the same reference on one host thread (a smaller sample)
            one = min(sample, 50_000)
            one_out, one_ms, _, _ = cpu_reference_rays(cfg.tris, cfg.rays[:one], 1)
            if int((one_out != result[:one]).sum()):
                raise RuntimeError("single-thread CPU reference differs")
            cpu["single_thread"] = {"value": round(one / (one_ms * 1e-3) / 1e6, 4),
                                    "unit": "Mrays/s", "cores": 1,
                                    "sample": f"first {one} rays, BVH build excluded"}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "median_ms_per_step": round(float(np.median(step_ms)), 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generators, identical bytes on every host)",
            "config": {**desc, "builder": best_builder, "sah_bins": 32, "variant": best,
                       "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": f"replica x{world}, rays sharded per rank"},
            "variants_ms": {k: round(v, 4) for k, v in results.items()},
            "build_ms": {k: round(v, 3) for k, v in build_ms.items()},
            "knn": {"k": 8, "queries": int(q_d.shape[0]), "ms": round(knn_ms, 4),
                    "variant": knn_variant,
                    "variants_ms": {kk: round(v, 4) for kk, v in knn_ms_by.items()},
                    "mqueries_per_s": round(q_d.shape[0] / (knn_ms * 1e-3) / 1e6, 2)},
            "fingerprint": f"0x{fp:016x}", "hits": int(hits), "parity": parity,
            "topology": topology,
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(cfg.rays.nbytes),
                    "d2h_bytes_per_step": int(nrays * 8),
                    "path": (f"qk_raycast_mapped, {e2e_pick}: the traversal reads pinned "
                             "host rays and writes pinned host results" if chunks == 0 else
                             f"qk_raycast_host, {e2e_pick}: uploads, traversals alternating "
                             "over two streams, "
                             + ("results stored by the traversals into pinned host memory"
                                if chunks < 0 else "read-backs, pinned host buffers")),
                    "flags": e2e_flags,
                    "chunks_ms": {k: round(v, 4) for k, v in chunk_ms.items()}},
            "gpu_launches": None,
        }
        # kernels of ours launched per timed step: Morton = reset + bounds + keys + 4 sort
        # passes x 5 + traversal; coherent = grid + keys + scan + scatter + traversal
        per_step = 1
        if best_flags & capi.QK_ORDER_MORTON:
            per_step = 3 + 4 * 5 + 1
        elif best_flags & capi.QK_ORDER_COHERENT:
            per_step = 4 + 1
        line["gpu_launches"] = args.steps * per_step
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
