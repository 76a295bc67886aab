"""Benchmark of the B200 spatial-query engine over its five benchmark configurations.

Default run (`python bench.py`): the city configuration is the headline line and the other
four ride along on the same JSON line under "configs":
  city     131,072 floorless box buildings (1,310,720 triangles) on a 363 x 362 lot grid,
           1,000,000 rays from a plane 50 units above the tallest roof with cosine-weighted
           downward directions, 20,000 kNN (k=8) queries uniform in the bounds
  terrain  256 x 256 height field (131,072 triangles), 1,000,000 rays straight down from
           z = +100, 20,000 closest-point queries in the bounds padded by 2; LBVH
  points   1,048,576 points on a noisy sphere and 1,048,576 uniform in [0,100]^3, 20,000
           queries each for closest / kNN8 / radius 1.0, and a coherent 1% refit
  grad     1,048,576 Gaussians x 262,144 queries, loss = sum of ellipsoid distances, and
           1,000,000 terrain rays, loss = sum of first-hit t, through quarry.torch's
           autograd functions (forward + backward)
  batch    256 uneven scenes (128 terrains of 1k..500k triangles, 128 uniform clouds of
           4k..1M points, 1k..100k queries each) in one CUDA graph per step vs the per-scene
           launch loop
Inputs are seeded synthetic data (quarry.workloads, the same bytes on every host).

A step of the headline is one pass of the hot path over resident inputs: trace the 1M rays
(the fastest of the engine's bit-identical variants).  `value` is rays per second over the
timed steps (CUDA events, L2 flushed between steps); `e2e` the same through the C ABI from
pinned host buffers with the 32 MB upload and 8 MB read-back inside the timed region.
Every ray and query result of every configuration is compared, outside the timed regions,
with quarry's own CPU reference (oracle/_ref): every unit, element for element, with both
FNV-1a fingerprints printed (each folded by the reference's own RayStats / QueryStats code).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload all|city|terrain|points|grad|batch] [--small]

Multi-GPU: one process per GPU (torchrun); every rank builds its own replica of the scene
and traces its own 1M rays (seed + rank; weak scaling, no data-path collective); time = max
over ranks.  The four extra configurations run at N = 1 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor
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
                    help="timed steps (default 400; the batch configuration times at most 20)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="all",
                    choices=["all", "city", "terrain", "grad", "batch", "points"])
    ap.add_argument("--tune-cache", default=None, help="autotuner JSON (default: user cache)")
    ap.add_argument("--retune", action="store_true", help="ignore cached autotuner choices")
    ap.add_argument("--small", action="store_true", help="small inputs (profiling captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU reference (parity checks and CPU timings)")
    ap.add_argument("--only", default="", help="time only this ray variant (profiling)")
    ap.add_argument("--dump", default="", help="also write the inputs as QRYD / QRCD files "
                                                "into this directory (for other engines)")
    ap.add_argument("--kernel-case", default="", choices=[""] + sorted(KERNEL_CASES),
                    help="run one kernel family twice on its configuration's inputs and exit "
                         "(no timing line): the target of a profiler capture")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 20 if args.workload == "batch" else 400
    args.warmup = max(args.warmup, 3)
    return args


def profiled_traffic(workload: str, variant: str) -> dict | None:
    """DRAM / L2 bytes of one launch of this variant's kernel (ncu, profiles/traffic.json)."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    return json.loads(p.read_text()).get(workload, {}).get(variant)


def peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return PEAKS_FALLBACK, "fallback"


def cpu_threads(world: int = 1) -> int:
    return max(1, (os.cpu_count() or 1) // max(1, world))


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


def morton_order(rays: np.ndarray) -> np.ndarray:
    """The engine's Morton ray order (30-bit origin codes, quarry's quantize10,
    src/gpu/morton.h), recomputed on the host."""
    o = rays[:, :3]
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
    return np.argsort(code, kind="stable")


def make_workload(w, name: str, small: bool, rank: int):
    """The city or terrain configuration from the workload module `w`; each rank traces its
    own rays (seed 1 + rank) over its own replica of the same scene.  The description is the
    `config` of both the engine's line and the reference arm's line."""
    seed = 1 + rank
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
                "rays": nr, "closest_queries": 20_000, "build": "lbvh"}
    return cfg, desc


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons around the timed region (every
    50 ms; the caller keeps the GPU loaded for a while before and after the timed steps)."""

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
                 "--format=csv,noheader,nounits", "-lms", "50"],
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


def loaded(fn, seconds: float) -> None:
    """Runs `fn` back to back for about `seconds` (keeps the clocks at their loaded state
    while the sampler runs)."""
    import torch

    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        for _ in range(8):
            fn()
        torch.cuda.synchronize()


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
# the reference arm: quarry's CPU implementation of the headline configuration
# ---------------------------------------------------------------------------------------
def reference_arm(args):
    """--impl reference: quarry's own CPU BVH (buildBVH + raycastBVH, src/cpu/bvh.cpp:91-178,
    compiled from its sources into oracle/_ref) tracing every ray of the headline
    configuration on all host threads.  Inputs come from the generators built on their own
    (oracle/_build/libqscenes.so), so this process loads no library of the engine.  Rank 0
    alone runs; other ranks exit at once."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import oracle

    w = oracle.standalone_workloads()
    name = "terrain" if args.workload == "terrain" else "city"
    cfg, desc = make_workload(w, name, args.small, 0)
    threads = cpu_threads()
    nrays = cfg.rays.shape[0]
    have_ref = oracle.ref_available()
    R = oracle.Reference() if have_ref else None
    port = None if have_ref else oracle.LBVH("tri", cfg.tris)
    times, out, build_ms = [], None, 0.0
    for i in range(args.warmup + args.steps):
        if R is not None:
            out, ms, build_ms = R.raycast(cfg.tris, cfg.rays, threads)
        else:
            t0 = time.perf_counter()
            out = port.raycast(cfg.rays, threads)
            ms = (time.perf_counter() - t0) * 1e3
        if i >= args.warmup:
            times.append(ms)
    ms = float(np.mean(times))
    value = nrays / (ms * 1e-3) / 1e6
    fp, hits = (R.ray_hash(out) if R is not None else oracle.ray_hash(out))
    kind = "reference" if have_ref else "port"
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
            "config": desc,
            "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads,
                             "kind": kind,
                             "sample": f"all {nrays} rays of the configuration per step; the "
                                       f"reference BVH ({build_ms:.0f} ms to build) is built "
                                       f"before each step, outside its time"},
            "fingerprint": f"0x{fp:016x}", "hits": int(hits),
            "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# rays: city (headline) and terrain
# ---------------------------------------------------------------------------------------
def l2_copy_peak(dev) -> dict:
    """L2 bandwidth the way MEASURED_PEAKS measures HBM: a device copy (read + write bytes per
    second, CUDA events) of a 32 MB buffer into another, both L2-resident (64 MB of the
    126 MB L2), best of 5 runs of 200 back-to-back copies."""
    import torch

    n = 8 * 1024 * 1024
    a = torch.ones(n, dtype=torch.float32, device=dev)
    b = torch.empty_like(a)
    for _ in range(20):
        b.copy_(a)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(200):
            b.copy_(a)
        e1.record()
        torch.cuda.synchronize()
        gbs = 200 * 2 * a.numel() * 4 / (e0.elapsed_time(e1) * 1e-3) / 1e9
        best = max(best, gbs)
    return {"gbs": round(best, 1), "how": "torch copy of 32 MB into 32 MB (L2-resident), "
                                         "read + write bytes, best of 5 x 200 copies"}


def rays_arm(args, world, rank, local, workload):
    """City or terrain: rays through the engine (the timed step), the configuration's point
    queries beside it, every result checked against quarry's CPU reference."""
    import torch

    import oracle
    from quarry import capi
    from quarry import workloads as w

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfg, desc = make_workload(w, workload, args.small, rank)
    city = workload == "city"
    nrays = cfg.rays.shape[0]
    if args.dump and rank == 0:
        from quarry import dumps

        Path(args.dump).mkdir(parents=True, exist_ok=True)
        dumps.write_qryd(Path(args.dump) / f"{workload}.qryd", cfg.tris, cfg.queries)

    # ---- builds (timed beside the step): LBVH, binned SAH with 32 bins, and the leaf-size-4
    # SAH (whose 4-wide nodes are the leaf-size-4 form) ----
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
        tr.build_wide(leaf4=builder == "sah4")
        return tr, float(np.median(times))

    trees, build_ms = {}, {}
    for b in ("lbvh", "sah", "sah4"):
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

    def time_variant(tree, flags, steps, warmup, clocks_window=0.0):
        out = torch.empty(nrays, dtype=torch.int64, device=dev)
        ws = torch.empty(capi.lib().qk_query_workspace_bytes(nrays, flags), dtype=torch.uint8,
                         device=dev)

        def one():
            tree.raycast(rays_d, flags, out=out, ws=ws)

        for _ in range(warmup):
            one()
        if clocks_window:
            loaded(one, clocks_window)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for e0, e1 in ev:
            l2_flush.zero_()
            e0.record()
            one()
            e1.record()
        torch.cuda.synchronize()
        if clocks_window:
            loaded(one, clocks_window / 3)
        return [e0.elapsed_time(e1) for e0, e1 in ev]

    results = {}
    for name, (b, flags) in variants.items():
        results[name] = float(np.median(time_variant(trees[b], flags, 10, 3)))
    # the city compares builders (the fastest variant of either); the terrain configuration
    # is specified with an LBVH, so its headline is the fastest LBVH variant
    pool = results if city or args.only else {k: v for k, v in results.items()
                                              if k.startswith("lbvh_")}
    best = min(pool, key=pool.get)
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
        step_ms = time_variant(tree, best_flags, args.steps, args.warmup, clocks_window=1.0)
    clocks = clk.summary()
    clocks["load"] = "the same step back to back for 1 s before and 0.3 s after the timed steps"
    ms = float(np.sum(step_ms)) / args.steps
    ms = max_over_ranks(world, ms)
    value = world * nrays / (ms * 1e-3) / 1e6

    # ---- roofline: traversal kernel alone on pre-sorted rays ----
    trav_flags = best_flags & ~(capi.QK_ORDER_MORTON | capi.QK_ORDER_COHERENT)
    if best_flags & capi.QK_ORDER_COHERENT:
        sorted_rays = capi.to_device(cfg.rays[coherent_order(cfg.rays)], np.float32)
    elif best_flags & capi.QK_ORDER_MORTON:
        sorted_rays = capi.to_device(cfg.rays[morton_order(cfg.rays)], np.float32)
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
    prof = profiled_traffic(workload, best) or {}
    l2peak = l2_copy_peak(dev)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4),
                "traffic": prof.get("dram_bytes"), "peak_kind": pk_kind,
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
    if prof.get("dram_bytes"):
        dram = prof["dram_bytes"] / (kernel_ms * 1e-3) / 1e9
        roofline["dram"] = {"bytes_per_launch": prof["dram_bytes"], "achieved_gbs": round(dram, 1),
                            "frac": round(dram / pk["hbm_gbs"], 4),
                            "source": prof.get("summary") or "profiles/traffic.json"}
    if prof.get("lts_bytes"):
        l2 = prof["lts_bytes"] / (kernel_ms * 1e-3) / 1e9
        roofline["l2"] = {"bytes_per_launch": prof["lts_bytes"], "achieved_gbs": round(l2, 1),
                          "peak_gbs": l2peak["gbs"], "frac": round(l2 / l2peak["gbs"], 4),
                          "peak_how": l2peak["how"],
                          "ncu_lts_pct_of_peak": prof.get("lts_pct_of_peak")}
    roofline["bound_met"] = (
        "dependent-load latency and issue: canonical bytes count every visited node at 96 B; "
        "the hot levels of the tree stay in L2, so DRAM and L2 carry far less than the "
        "canonical bytes and neither bandwidth is near its peak")

    # ---- the configuration's point queries: kNN8 (city) or closest (terrain) ----
    qname = "knn" if city else "closest"

    def query(flags, out_t=None):
        return tree.knn(q_d, 8, flags, out=out_t) if city else tree.closest(q_d, flags, out=out_t)

    q_base = (trees["lbvh"].knn(q_d, 8, 0) if city else trees["lbvh"].closest(q_d, 0)).clone()
    q_out = torch.empty_like(q_base)
    q_ms_by = {}
    for kname, kf in (("layout_of_rays", best_flags & (capi.QK_WIDE | capi.QK_ORDER_MORTON |
                                                       capi.QK_ORDER_COHERENT)),
                      ("input", 0), ("morton", capi.QK_ORDER_MORTON),
                      ("coherent", capi.QK_ORDER_COHERENT),
                      ("split", capi.QK_TUNE_SPLIT),
                      ("split_morton", capi.QK_TUNE_SPLIT | capi.QK_ORDER_MORTON),
                      ("split_coherent", capi.QK_TUNE_SPLIT | capi.QK_ORDER_COHERENT),
                      ("split8", capi.QK_TUNE_SPLIT8),
                      ("split8_coherent", capi.QK_TUNE_SPLIT8 | capi.QK_ORDER_COHERENT),
                      ("split4", capi.QK_TUNE_SPLIT4),
                      ("split4_coherent", capi.QK_TUNE_SPLIT4 | capi.QK_ORDER_COHERENT),
                      ("leaf4", capi.QK_TUNE_LEAF4),
                      ("leaf4_morton", capi.QK_TUNE_LEAF4 | capi.QK_ORDER_MORTON)):
        for _ in range(3):
            query(kf, q_out)
        if not torch.equal(q_out, q_base):
            raise RuntimeError(f"{qname} variant {kname} differs")
        qt = []
        for _ in range(10):
            l2_flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            query(kf, q_out)
            e1.record()
            torch.cuda.synchronize()
            qt.append(e0.elapsed_time(e1))
        q_ms_by[kname] = float(np.median(qt))
    q_variant = min(q_ms_by, key=q_ms_by.get)
    q_ms = q_ms_by[q_variant]
    q_result = q_base.cpu().numpy().view(np.uint32)

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
    if city:
        topology = topology_timing("tri", cfg.tris, "sah", 32, q_d, 1 + rank, med_ms,
                                   rays_d[:200_000])

    # ---- e2e through the C ABI from pinned host buffers: qk_raycast_host uploads, traces and
    # reads back in chunks (uploads, traversals and read-backs on separate streams), all inside
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
    if not np.array_equal(host_out.numpy(), base.cpu().numpy()):
        raise RuntimeError("e2e results differ from the device-resident run")
    e2e_ms = max_over_ranks(world, float(np.mean(e2e_t)))
    e2e_value = world * nrays / (e2e_ms * 1e-3) / 1e6

    result = host_out.numpy().view(np.uint64)

    # ---- every ray and every query against quarry's CPU reference (each rank its own) ----
    parity, cpu = None, None
    if not args.no_cpu_baseline:
        parity, cpu = rays_parity(cfg, result, q_result, city, cpu_threads(world), rank == 0)

    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "median_ms_per_step": round(float(np.median(step_ms)), 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators, identical bytes on every host)",
        "config": desc,
        "engine": {"builder": best_builder, "sah_bins": 32, "variant": best,
                   "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": (f"{world} rank(s); each builds its own replica of the scene "
                                   f"and traces its own {nrays} rays (weak scaling)")},
        "variants_ms": {k: round(v, 4) for k, v in results.items()},
        "build_ms": {k: round(v, 3) for k, v in build_ms.items()},
        qname: {"k": 8, "queries": int(q_d.shape[0]), "ms": round(q_ms, 4)} if city else
        {"queries": int(q_d.shape[0]), "ms": round(q_ms, 4)},
        "parity": parity, "topology": topology,
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
    line[qname].update({"variant": q_variant,
                        "variants_ms": {kk: round(v, 4) for kk, v in q_ms_by.items()},
                        "mqueries_per_s": round(q_d.shape[0] / (q_ms * 1e-3) / 1e6, 2)})
    if not city:
        sah = {k: v for k, v in results.items() if k.startswith("sah_")}
        sbest = min(sah, key=sah.get)
        line["sah_tree"] = {"variant": sbest, "ms": round(sah[sbest], 4),
                            "mrays_per_s": round(nrays / (sah[sbest] * 1e-3) / 1e6, 1),
                            "note": "same bits; SAH tree instead of the configuration's LBVH"}
    # kernels of ours launched per timed step: Morton = reset + bounds + keys + 4 sort
    # passes x 5 + traversal; coherent = grid + keys + scan + scatter + traversal
    per_step = 1
    if best_flags & capi.QK_ORDER_MORTON:
        per_step = 3 + 4 * 5 + 1
    elif best_flags & capi.QK_ORDER_COHERENT:
        per_step = 4 + 1
    line["gpu_launches"] = args.steps * per_step
    return line


def rays_parity(cfg, result, q_result, city: bool, threads: int, report_cpu: bool):
    """Every ray (and every kNN8 / closest query) of the configuration against quarry's CPU
    reference, element for element; both fingerprints folded by the reference's own code.
    Also times the reference (the CPU baseline: every ray on `threads` host threads, and a
    50,000-ray sample on one thread)."""
    import oracle

    nrays = cfg.rays.shape[0]
    have_ref = oracle.ref_available()
    if have_ref:
        R = oracle.Reference()
        ref_rays, ref_ms, ref_build = R.raycast(cfg.tris, cfg.rays, threads)
        if city:
            ref_q, _, _ = R.knn("tri", cfg.tris, cfg.queries, 8, threads)
        else:
            ref_q, _, _ = R.closest("tri", cfg.tris, cfg.queries, threads)
        fold_rays, fold_closest = R.ray_hash, R.closest_hash

        def fold_knn(res):
            return R.list_hash(*oracle.knn_to_csr(res))
    else:
        ref = oracle.LBVH("tri", cfg.tris)
        t0 = time.perf_counter()
        ref_rays = ref.raycast(cfg.rays, threads)
        ref_ms, ref_build = (time.perf_counter() - t0) * 1e3, 0.0
        ref_q = ref.knn(cfg.queries, 8, threads) if city else ref.closest(cfg.queries, threads)
        fold_rays, fold_closest, fold_knn = oracle.ray_hash, oracle.closest_hash, oracle.knn_hash
    kind = "reference" if have_ref else "port"
    mism = int((ref_rays != result).sum())
    q_want = ref_q.reshape(q_result.shape)
    q_mism = int((q_want != q_result).reshape(q_result.shape[0], -1).any(axis=1).sum())
    (fe, he), (fr, hr) = fold_rays(result), fold_rays(ref_rays)
    qfold = fold_knn if city else fold_closest
    qe, qr = qfold(q_result), qfold(q_want)
    parity = {"against": kind,
              "rays": {"checked": nrays, "mismatches": mism, "fingerprint": f"0x{fe:016x}",
                       "reference_fingerprint": f"0x{fr:016x}", "hits": int(he),
                       "reference_hits": int(hr)},
              ("knn" if city else "closest"): {
                  "checked": int(q_result.shape[0]), "mismatches": q_mism,
                  "fingerprint": f"0x{qe:016x}", "reference_fingerprint": f"0x{qr:016x}"}}
    if mism or q_mism or fe != fr or qe != qr:
        raise RuntimeError(f"results differ from the CPU reference: {parity}")
    if not report_cpu:
        return parity, None
    cpu = {"value": round(nrays / (ref_ms * 1e-3) / 1e6, 4), "unit": "Mrays/s",
           "cores": threads, "kind": kind,
           "sample": f"all {nrays} rays of the step (the parity run), reference BVH build "
                     f"({ref_build:.0f} ms) excluded"}
    if have_ref:
        one = min(nrays, 50_000)
        one_out, one_ms, _ = R.raycast(cfg.tris, cfg.rays[:one], 1)
        if int((one_out != result[:one]).sum()):
            raise RuntimeError("single-thread CPU reference differs")
        cpu["single_thread"] = {"value": round(one / (one_ms * 1e-3) / 1e6, 4),
                                "unit": "Mrays/s", "cores": 1,
                                "sample": f"first {one} rays, BVH build excluded"}
    return parity, cpu


# ---------------------------------------------------------------------------------------
# topology edits: subtree surgery against a rebuild of the edited scene
# ---------------------------------------------------------------------------------------
def topology_surgery(kind, items, builder, bins, mode, seed):
    """A 1% edit script of quarry's GpuTopoEdit kind (a quarter each deleted, inserted,
    appended and moved; "cluster" around one spot or "scatter" uniform) for a tree built from
    `items`: returns the tree, the edited scene and the script on the device, the QkTopoInfo
    the surgery fills and a function that runs qk_update_topology once on the built tree."""
    import ctypes

    import torch

    from quarry import capi
    from quarry import workloads as w

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
    keep = (dele_d, ins_d, mov_d, extra, moved_items, arrays, nt, ws, e)

    def surgery():
        capi.check(capi.lib().qk_update_topology(
            ctypes.byref(base.t), ctypes.byref(nt), ctypes.byref(e), 0, bins,
            ctypes.byref(info), ws.data_ptr(), nb, capi._stream()), "qk_update_topology")

    script = (new, dele, ins, mov, int(len(dele) + len(ins) + app + len(mov)))
    return base, new_d, script, info, surgery, keep


def topology_timing(kind, items, builder, bins, queries_d, seed, timed_ms, rays_d=None):
    """1% edits of quarry's GpuTopoEdit kind (a quarter each deleted, inserted, appended and
    moved), "cluster" (around one spot) and "scatter" (uniform): qk_update_topology on the
    built tree against qk_build of the edited scene, both device-timed with the scripts
    already resident.  The edited tree must answer closest / kNN (and rays) like the rebuild."""
    import torch

    from quarry import capi

    out = {}
    for mode in ("cluster", "scatter"):
        base, new_d, script, info, surgery, keep = topology_surgery(kind, items, builder, bins,
                                                                    mode, seed)
        new, dele, ins, mov, edited = script
        s_ms = timed_ms(surgery)
        fresh = capi.DeviceTree(kind, new_d, builder=builder, sah_bins=bins)
        b_ms = timed_ms(fresh.build)
        entry = {"edited": edited, "surgery_ms": round(s_ms, 4),
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
        del base, fresh, keep
    return out


def topology_api_wall(kind, items, new, dele, ins, mov, builder, rounds=4):
    """Host wall time through the module (the C++ updateBVHGPU: it uploads only the edit
    script and the primitives it brings, and reuses its arrays from the previous edit) in
    steady state -- one object takes `rounds` further 1% edits of the same kind after the first
    (which allocates), the later ones timed -- against constructing the object from the whole
    edited scene (conversion, allocation, upload, build).  Medians."""
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
    stages = []
    for r in range(rounds):
        nxt, d2, i2, m2 = w.topology_edit(cur, 0.01, "cluster", 100 + r)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tm = obj.update_topology(wrap(nxt), deleted=d2, moved=m2, inserted=i2)
        upd.append((time.perf_counter() - t0) * 1e3)
        inner.append(float(tm["total_ms"]))
        stages.append({k: float(tm[k]) for k in ("plan_ms", "relayout_ms", "surgery_ms",
                                                 "merge_ms") if k in tm})
        full += int(bool(tm["full_rebuild"]))
        t0 = time.perf_counter()
        fresh = make(nxt)
        reb.append((time.perf_counter() - t0) * 1e3)
        del fresh
        cur = nxt
    u, r = float(np.median(upd[1:])), float(np.median(reb[1:]))
    out = {"update_wall_ms": round(u, 3), "rebuild_wall_ms": round(r, 3), "ratio": round(u / r, 3),
           "update_cpp_total_ms": round(float(np.median(inner[1:])), 3),
           "full_rebuilds": full, "rounds": rounds, "timed": "rounds 2..n, cluster 1% each",
           "note": "walls include the module's host conversion of the whole scene (both paths)"}
    if stages and stages[-1]:
        out["update_stages_ms"] = {k: round(float(np.median([s[k] for s in stages[1:]])), 4)
                                   for k in stages[-1]}
    return out


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
    from quarry import capi
    from quarry import workloads as w

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
        for bname, builder, bins in (("lbvh", "lbvh", 32), ("sah8", "sah", 8), ("sah32", "sah", 32),
                                     ("sah4", "sah4", 32)):
            trees[bname] = capi.DeviceTree("point", pts, builder=builder, sah_bins=bins)
            # the leaf-size-4 SAH tree carries the leaf-size-4 4-wide form
            trees[bname].build_wide(leaf4=builder == "sah4")
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
                "split8": capi.QK_TUNE_SPLIT8, "split8_coh": capi.QK_TUNE_SPLIT8 | capi.QK_ORDER_COHERENT,
                "split4": capi.QK_TUNE_SPLIT4, "split4_coh": capi.QK_TUNE_SPLIT4 | capi.QK_ORDER_COHERENT,
                "leaf4_coh": capi.QK_TUNE_LEAF4 | capi.QK_ORDER_COHERENT}
    # the heavy-query tail (closest / kNN): shell queries near the centre go to the shared scan
    tail = capi.QK_TUNE_TAIL
    tail_variants = {"bin_tail": tail, "bin_coh_tail": tail | capi.QK_ORDER_COHERENT,
                     "split_tail": capi.QK_TUNE_SPLIT | tail,
                     "split_coh_tail": capi.QK_TUNE_SPLIT | capi.QK_ORDER_COHERENT | tail}
    radius_variants = {"stash": capi.QK_TUNE_STASH,
                       "stash_morton": capi.QK_TUNE_STASH | capi.QK_ORDER_MORTON,
                       "stash_leaf4": capi.QK_TUNE_STASH | capi.QK_TUNE_LEAF4,
                       "stash_coh": capi.QK_TUNE_STASH | capi.QK_ORDER_COHERENT}
    vms, plan = {}, {}
    for kind, c in clouds.items():
        for op in ops:
            run(kind, op, c["trees"]["lbvh"], 0)
            base = snapshot((kind, op))
            cands = ({**variants, **radius_variants} if op == "radius" else
                     {**variants, **tail_variants})
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
    variants.update(tail_variants)

    def step():
        for (kind, op), (bname, vname, _) in plan.items():
            run(kind, op, clouds[kind]["trees"][bname], variants[vname])

    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        loaded(step, 0.5)
        ts = timed(step, args.steps, args.warmup)
        loaded(step, 0.2)
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
        split = f & (capi.QK_TUNE_SPLIT | capi.QK_TUNE_SPLIT8 | capi.QK_TUNE_SPLIT4)
        return ("k_%s_wide" if f & capi.QK_WIDE else "k_%s_split" if split else "k_%s_bin") % op

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
        if flip[0] % 2 == 0:  # leave the tree on the moved points
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

    # quarry's CPU reference on every query of the step, all host threads
    threads = cpu_threads(world)
    parity, cpu_ms, kind_ref = {}, 0.0, "port"
    if not args.no_cpu_baseline:
        R = oracle.Reference() if oracle.ref_available() else None
        kind_ref = "reference" if R is not None else "port"
        for kind, c in clouds.items():
            if R is not None:
                cw, cms, _ = R.closest("point", c["pts"], c["q"], threads)
                kw_, kms, _ = R.knn("point", c["pts"], c["q"], k, threads)
                ro, rk, rms = R.radius("point", c["pts"], c["q"], r, threads)
            else:
                ref = oracle.LBVH("point", c["pts"])
                t0 = time.perf_counter()
                cw, kw_ = ref.closest(c["q"], threads), ref.knn(c["q"], k, threads)
                ro, rk = ref.radius(c["q"], r, threads)
                cms, kms, rms = (time.perf_counter() - t0) * 1e3, 0.0, 0.0
            cpu_ms += cms + kms + rms
            got_c = outs[(kind, "closest")].cpu().numpy().view(np.uint32)
            got_k = outs[(kind, "knn")].cpu().numpy().view(np.uint32)
            got_o = outs[(kind, "radius")][0].cpu().numpy().astype(np.int64)
            got_r = outs[(kind, "radius")][1].cpu().numpy().view(np.uint64)
            mism = {"closest": int((got_c != cw).any(axis=1).sum()),
                    "knn": int((got_k != kw_).reshape(nq, -1).any(axis=1).sum()),
                    "radius_offsets": int((got_o != ro).sum()),
                    "radius_keys": int(got_r.size != rk.size or (got_r != rk).sum())}
            fold_l = (R.list_hash if R is not None else oracle.radius_hash)
            fold_c = (R.closest_hash if R is not None else oracle.closest_hash)
            fps = {"closest": (fold_c(got_c), fold_c(cw)),
                   "knn": (fold_l(*oracle.knn_to_csr(got_k)), fold_l(*oracle.knn_to_csr(kw_))),
                   "radius": (fold_l(got_o, got_r), fold_l(ro, rk))}
            parity[kind] = {"queries_per_op": nq, "mismatches": mism,
                            "fingerprints": {op: f"0x{a:016x}" for op, (a, _) in fps.items()},
                            "reference_fingerprints": {op: f"0x{b:016x}"
                                                       for op, (_, b) in fps.items()}}
            if any(mism.values()) or any(a != b for a, b in fps.values()):
                raise RuntimeError(f"{kind}: results differ from the CPU reference: {parity[kind]}")

    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mqueries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators, identical bytes on every host)",
        "config": {"workload": "points", "points_per_cloud": n, "clouds": ["surface", "volume"],
                   "queries_per_op": nq, "k": k, "radius": r},
        "engine": {"plan": {f"{kind}/{op}": f"{b}/{v}" for (kind, op), (b, v, _) in plan.items()},
                   "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"{world} rank(s), each its own replica of both clouds"},
        "variants_ms": {kk: round(v, 4) for kk, v in vms.items()},
        "per_op_ms": {kk: round(v, 4) for kk, v in per_op.items()},
        "radius_results": radius_keys, "refit": refit, "topology": topology,
        "parity": {"against": kind_ref, "clouds": parity,
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
        # scan + merge for each round of up to 1,024 queries past the budget (one round here)
        tail_k = 2 if variants[vname] & capi.QK_TUNE_TAIL else 0
        launches += (1 + morton + tail_k) if op != "radius" else (4 + morton) + (1 + morton) + 4
    line["gpu_launches"] = args.steps * launches
    return line


# ---------------------------------------------------------------------------------------
# differentiable queries through quarry.torch: forward and forward + backward
# ---------------------------------------------------------------------------------------
def grad_arm(args, world, rank, local):
    """1,048,576 Gaussians (means U[0,100]^3, log-uniform scales [0.05, 1], random rotations)
    with 262,144 query points, loss = sum of point-to-ellipsoid distances, gradients to the
    points, means, quaternions and scales; and 1M downward rays on the 256 x 256 terrain
    (shared vertices), loss = sum of first-hit t, gradients to the vertices.  Both run through
    quarry.torch's autograd functions as a caller would (the forward builds the tree from the
    current parameters; the backward includes the per-vertex segmented sum).  Checked against
    FP64 analytic gradients of every output and FP64 central differences on 1,000 parameters
    of each part, at full size."""
    import torch

    import quarry.torch as qt
    from quarry import capi
    from quarry import workloads as w

    torch.cuda.set_device(local)
    small = args.small
    ng, nq = (65_536, 16_384) if small else (1_048_576, 262_144)
    g = w.gaussians(ng, 0.05, 1.0, 1 + rank)
    q = w.uniform_points(nq, [0, 0, 0], [100, 100, 100], 1 + rank, 31)
    G = torch.tensor(g, device="cuda")
    pts = torch.tensor(q, device="cuda", requires_grad=True)
    means = G[:, 0:3].clone().requires_grad_(True)
    rots = G[:, 3:7].clone().requires_grad_(True)
    scales = G[:, 7:10].clone().requires_grad_(True)
    params = (pts, means, rots, scales)
    l2 = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def fwd_bwd_times(fwd, steps, warm=3):
        """(forward ms, backward ms) medians: forward = the autograd function's forward (tree
        build + query), backward = loss.backward() (adjoint kernels + the sums autograd does)."""
        for _ in range(warm):
            fwd().sum().backward()
        f, b = [], []
        for _ in range(steps):
            for p in params + tri_params:
                p.grad = None
            l2.zero_()
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record()
            out = fwd()
            e[1].record()
            loss = out.sum()
            e[2].record()
            loss.backward()
            e[3].record()
            torch.cuda.synchronize()
            f.append(e[0].elapsed_time(e[1]))
            b.append(e[2].elapsed_time(e[3]))
        return float(np.median(f)), float(np.median(b))

    # triangles: the terrain as shared vertices + indices, 1M rays straight down
    grid = 64 if small else 256
    tris = w.terrain(grid, 1)
    verts, inv = np.unique(tris.reshape(-1, 3), axis=0, return_inverse=True)
    idx = inv.reshape(-1, 3).astype(np.int32)
    nr = 100_000 if small else 1_000_000
    rays = w.down_rays(nr, 0.0, float(grid), 0.0, float(grid), 100.0, 1 + rank)
    V = torch.tensor(verts.astype(np.float32), device="cuda", requires_grad=True)
    I = torch.tensor(idx, device="cuda")
    O = torch.tensor(rays[:, 0:3], device="cuda", requires_grad=True)
    D = torch.tensor(rays[:, 3:6], device="cuda", requires_grad=True)
    tri_params = (V, O, D)

    # forward schedule (order, layout) chosen by measurement; all give the same bits
    g_opts = {"morton": ("morton", False), "coherent": ("coherent", False),
              "wide_coherent": ("coherent", True), "input": ("input", False)}
    g_by, g_ref = {}, None
    for name, (order, wide) in g_opts.items():
        d = qt.gaussian_distance(pts, means, rots, scales, order=order, wide=wide).detach()
        if g_ref is None:
            g_ref = d.clone()
        elif not torch.equal(d, g_ref):
            raise RuntimeError(f"gaussian forward {name} differs")
        g_by[name] = fwd_bwd_times(lambda o=order, wd=wide: qt.gaussian_distance(
            pts, means, rots, scales, order=o, wide=wd), 3)
    g_pick = min(g_by, key=lambda k: g_by[k][0])
    order, wide = g_opts[g_pick]
    g_fwd, g_bwd = fwd_bwd_times(lambda: qt.gaussian_distance(pts, means, rots, scales,
                                                              order=order, wide=wide), 10)

    r_opts = {"input": "input", "morton": "morton", "coherent": "coherent"}
    r_by, r_ref = {}, None
    for name, order_r in r_opts.items():
        t, hit = qt.ray_hit_t(O, D, V, I, order=order_r)
        if r_ref is None:
            r_ref = t.detach().clone()
        elif not torch.equal(t.detach(), r_ref):
            raise RuntimeError(f"ray forward {name} differs")
        r_by[name] = fwd_bwd_times(lambda o=order_r: qt.ray_hit_t(O, D, V, I, order=o)[0], 3)
    r_pick = min(r_by, key=lambda k: r_by[k][0])
    r_fwd, r_bwd = fwd_bwd_times(lambda: qt.ray_hit_t(O, D, V, I, order=r_pick)[0], 10)
    if not bool(torch.isfinite(r_ref).all()):
        raise RuntimeError("a terrain ray missed")

    # gradients of the timed passes' last step, then the checks (FP64, host)
    for p in params + tri_params:
        p.grad = None
    qt.gaussian_distance(pts, means, rots, scales, order=order, wide=wide).sum().backward()
    qt.ray_hit_t(O, D, V, I, order=r_pick)[0].sum().backward()
    checks = None
    if not args.no_cpu_baseline:
        tree = capi.DeviceTree("gauss", G)
        ids = tree.closest(pts.detach()).cpu().numpy()[:, 1].astype(np.int64)
        tri_tree = capi.DeviceTree("tri", tris)
        _, rid = tri_tree.raycast_ids(capi.to_device(rays, np.float32))
        checks = grad_checks(g, q, ids, pts.grad, means.grad, rots.grad, scales.grad,
                             verts, idx, rays, rid.cpu().numpy().astype(np.int64), V.grad,
                             O.grad, D.grad, g_ref.cpu().numpy(), r_ref.cpu().numpy(), rank)

    if rank != 0:
        return None
    line = {"metric": METRIC, "value": round((g_fwd + g_bwd) / g_fwd, 4),
            "unit": "fwd+bwd / fwd (Gaussian closest distance)", "n_gpus": world,
            "steps": 10, "warmup": 3, "ms_per_step": round(g_fwd + g_bwd, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 forward, f64 adjoint", "data": "synthetic (seeded generators)",
            "config": {"workload": "gaussian distance + ray t gradients", "gaussians": ng,
                       "queries": nq, "rays": nr, "terrain_grid": grid},
            "engine": {"path": "quarry.torch.gaussian_distance / ray_hit_t (autograd.Function); "
                               "forward = tree build + query, backward = loss.backward()",
                       "l2": "flushed between timed steps"},
            "gaussian": {"forward_ms": round(g_fwd, 4), "backward_ms": round(g_bwd, 4),
                         "fwd_bwd_over_fwd": round((g_fwd + g_bwd) / g_fwd, 4),
                         "forward_schedule": g_pick,
                         "schedules_ms": {k: [round(v[0], 4), round(v[1], 4)]
                                          for k, v in g_by.items()},
                         "mqueries_per_s_fwd": round(nq / (g_fwd * 1e-3) / 1e6, 2)},
            "rays": {"forward_ms": round(r_fwd, 4), "backward_ms": round(r_bwd, 4),
                     "fwd_bwd_over_fwd": round((r_fwd + r_bwd) / r_fwd, 4),
                     "order": r_pick,
                     "orders_ms": {k: [round(v[0], 4), round(v[1], 4)] for k, v in r_by.items()}},
            "checks": checks}
    return line


def grad_checks(g, q, ids, gp, gm, gr, gs, verts, idx, rays, rid, gv, go, gd, d_gpu, t_gpu,
                rank) -> dict:
    """Every gradient output against the FP64 analytic gradient (all queries / rays), and
    1,000 random parameters of each part against FP64 central differences (h = 1e-3) and
    their Richardson extrapolation, the forward's selection held fixed.  Relative errors
    |g - ref| / max(|ref|, 1e-3), stated per output."""
    from oracle import grad64 as G64

    rng = np.random.default_rng(11 + rank)
    out = {"floor": 1e-3, "h": G64.H}
    Gd, P = g.astype(np.float64), q.astype(np.float64)
    sel = ids >= 0
    if not sel.all():
        raise RuntimeError("a Gaussian query found nothing")
    dd, ref_p, ref_g = G64.gaussian_analytic(P, Gd, ids, iters=64)
    out["gaussian_forward_max_abs_err"] = float(np.max(np.abs(d_gpu - dd)))
    got = {"points": gp.cpu().numpy().astype(np.float64), "means": gm.cpu().numpy().astype(np.float64),
           "quaternions": gr.cpu().numpy().astype(np.float64),
           "scales": gs.cpu().numpy().astype(np.float64)}
    refs = {"points": ref_p, "means": ref_g[:, 0:3], "quaternions": ref_g[:, 3:7],
            "scales": ref_g[:, 7:10]}
    out["gaussian_analytic"] = {k: G64.fd_stats(G64.rel_err(got[k], refs[k], 1e-3).ravel())
                                for k in got}
    # normwise: max |g - ref| / max |ref| over each output
    for k in got:
        out["gaussian_analytic"][k]["normwise"] = float(
            np.max(np.abs(got[k] - refs[k])) / max(np.max(np.abs(refs[k])), 1e-30))
    # central differences: 250 coordinates of each input.  The distance has a kink at d = 0
    # (inside the solid it is 0), so a difference whose +-h step could carry a selected query
    # across the surface is not a reference: parameters whose queries lie within 1e-2 of
    # their ellipsoid (ten steps) are not drawn.
    order = np.argsort(ids, kind="stable")
    starts = np.searchsorted(ids[order], np.arange(len(g) + 1))
    near = np.zeros(len(g), bool)
    np.logical_or.at(near, ids, dd < 1e-2)
    used = np.unique(ids[dd > 0])
    used = used[~near[used]]
    fd_errs = {k: ([], []) for k in got}
    for k in got:
        for _ in range(250):
            if k == "points":
                i = int(rng.integers(len(q)))
                while dd[i] < 1e-2:
                    i = int(rng.integers(len(q)))
                c = int(rng.integers(3))

                def loss(delta, i=i, c=c):
                    p2 = P[i:i + 1].copy()
                    p2[0, c] += delta
                    return G64.ellipsoid_d(p2, Gd[ids[i]:ids[i] + 1], 80)[0].sum()
                val = got[k][i, c]
            else:
                gi = int(rng.choice(used))
                c = int(rng.integers({"means": 3, "quaternions": 4, "scales": 3}[k]))
                col = {"means": 0, "quaternions": 3, "scales": 7}[k] + c
                rows = order[starts[gi]:starts[gi + 1]]

                def loss(delta, gi=gi, col=col, rows=rows):
                    G2 = np.repeat(Gd[gi:gi + 1], len(rows), 0)
                    G2[:, col] += delta
                    return G64.ellipsoid_d(P[rows], G2, 80)[0].sum()
                val = got[k][gi, c]
            fd, rich = G64.central(loss)
            fd_errs[k][0].append(G64.rel_err(val, fd, 1e-3))
            fd_errs[k][1].append(G64.rel_err(val, rich, 1e-3))
    out["gaussian_fd"] = {k: {"central": G64.fd_stats(a), "richardson": G64.fd_stats(b)}
                          for k, (a, b) in fd_errs.items()}

    # rays: analytic for every ray, vertex sums; 1,000 vertex coordinates by differences
    Vd = verts.astype(np.float64)
    O, D = rays[:, 0:3].astype(np.float64), rays[:, 3:6].astype(np.float64)
    if (rid < 0).any():
        raise RuntimeError("a terrain ray missed")
    a, b, c = Vd[idx[rid, 0]], Vd[idx[rid, 1]], Vd[idx[rid, 2]]
    tt, wts, kk = G64.ray_analytic(O, D, a, b, c)
    out["ray_forward_max_abs_err"] = float(np.max(np.abs(t_gpu - tt)))
    ref_v = np.zeros_like(Vd)
    for j, wj in enumerate(wts):
        np.add.at(ref_v, idx[rid, j], wj[:, None] * kk)
    gvn = gv.cpu().numpy().astype(np.float64)
    pairs = {"vertices": (gvn, ref_v), "origins": (go.cpu().numpy().astype(np.float64), -kk),
             "directions": (gd.cpu().numpy().astype(np.float64), -tt[:, None] * kk)}
    out["ray_analytic"] = {}
    for k, (a_, r_) in pairs.items():
        st = G64.fd_stats(G64.rel_err(a_, r_, 1e-3).ravel())
        st["normwise"] = float(np.max(np.abs(a_ - r_)) / max(np.max(np.abs(r_)), 1e-30))
        out["ray_analytic"][k] = st
    vert_of = idx[rid].reshape(-1)
    vorder = np.argsort(vert_of, kind="stable")
    vstart = np.searchsorted(vert_of[vorder], np.arange(len(Vd) + 1))
    touched = np.unique(vert_of)
    e1, e2 = [], []
    for _ in range(1000):
        vi = int(rng.choice(touched))
        comp = int(rng.integers(3))
        rows = np.unique(vorder[vstart[vi]:vstart[vi + 1]] // 3)

        def loss(delta, vi=vi, comp=comp, rows=rows):
            tri = idx[rid[rows]]
            A, B, C = Vd[tri[:, 0]].copy(), Vd[tri[:, 1]].copy(), Vd[tri[:, 2]].copy()
            for arr, col in ((A, 0), (B, 1), (C, 2)):
                arr[tri[:, col] == vi, comp] += delta
            return G64.ray_t(O[rows], D[rows], A, B, C).sum()
        fd, rich = G64.central(loss)
        e1.append(G64.rel_err(gvn[vi, comp], fd, 1e-3))
        e2.append(G64.rel_err(gvn[vi, comp], rich, 1e-3))
    out["ray_fd_vertices"] = {"central": G64.fd_stats(e1), "richardson": G64.fd_stats(e2)}
    # the target (1e-4 against FP64 finite differences) on the Richardson-extrapolated
    # differences, and on the analytic gradient of every output normwise; elementwise figures
    # are reported beside them (an element whose terms cancel shows the FP32 rounding of the
    # per-primitive sums relative to its own small value)
    worst = max([v["richardson"]["max"] for v in out["gaussian_fd"].values()] +
                [out["ray_fd_vertices"]["richardson"]["max"]] +
                [v["normwise"] for v in out["gaussian_analytic"].values()] +
                [v["normwise"] for v in out["ray_analytic"].values()])
    out["max_rel_err"] = worst
    out["max_elementwise_rel_err"] = max([v["max"] for v in out["gaussian_analytic"].values()] +
                                         [v["max"] for v in out["ray_analytic"].values()])
    out["target"] = 1e-4
    if worst > 1e-4:
        raise RuntimeError(f"gradient error {worst:.3g} above 1e-4: {out}")
    return out


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
    from quarry import autotune, pipeline
    from quarry import workloads as w

    torch.cuda.set_device(local)
    kw = {}
    if args.small:
        kw = dict(terrains=16, clouds=16, tri_range=(1_000, 50_000),
                  point_range=(4_000, 100_000), query_range=(1_000, 10_000))
    steps = min(args.steps, 20)
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
    for _ in range(args.warmup):
        pipe.replay()
    torch.cuda.synchronize()
    pipe.sync()

    # ---- batched: K graph replays (inputs are GBs, larger than L2) ----
    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    with Clocks(local) as clk:
        loaded(pipe.replay, 0.5)
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
    for _ in range(min(steps, 5)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        e2e_step()
        e1.record()
        torch.cuda.synchronize()
        et.append(e0.elapsed_time(e1))
    e2e_ms = max_over_ranks(world, float(np.mean(et)))
    nq = pipe.query_count()

    # ---- every scene against quarry's CPU reference (one reference structure per scene,
    # scenes on parallel host threads) ----
    parity, cpu = None, None
    if not args.no_cpu_baseline:
        parity, cpu = batch_parity(cfg, got, cpu_threads(world))

    if rank != 0:
        return None
    speedup = loop_ms / batched_ms
    line = {
        "metric": METRIC, "value": round(speedup, 3), "unit": "x (per-scene loop / batched)",
        "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": round(batched_ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators, identical bytes on every host)",
        "config": {"workload": "batch", "scenes": len(cfg.terrains) + len(cfg.clouds),
                   "terrains": len(cfg.terrains), "clouds": len(cfg.clouds),
                   "triangles": int(sum(s.items.shape[0] for s in cfg.terrains)),
                   "points": int(sum(s.items.shape[0] for s in cfg.clouds)),
                   "queries": nq, "k": cfg.k,
                   "step": "build every tree + every query of every scene"},
        "engine": {"builder": pipe.builder,
                   "l2": "inputs and trees (GBs) larger than L2; no flush",
                   "parallelism": f"{world} rank(s), each its own 256 scenes"},
        "batched": {"ms": round(batched_ms, 3),
                    "mqueries_per_s": round(world * nq / (batched_ms * 1e-3) / 1e6, 2),
                    "graph_kernel_nodes": pipe.graph_kernel_nodes()},
        "loop": {"ms": round(loop_ms, 3), "steps": loop_steps,
                 "mqueries_per_s": round(world * nq / (loop_ms * 1e-3) / 1e6, 2)},
        "autotune": tune_report, "tune_cache": str(tuner.path),
        "parity": parity,
        "roofline": None,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "e2e": {"value": round(world * nq / (e2e_ms * 1e-3) / 1e6, 2), "unit": "Mqueries/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "pinned host inputs -> graph replay -> pinned host outputs"},
        "generate_s": round(gen_s, 1),
        "gpu_launches": (pipe.graph_kernel_nodes() or 0) * steps,
    }
    return line


def batch_parity(cfg, got, threads: int):
    """Every query and ray of every scene against quarry's CPU reference (oracle/_ref: one
    reference structure per scene, qr_scene), element for element, with per-scene fingerprints
    folded by the reference's code; scenes run concurrently on host threads."""
    import oracle

    have_ref = oracle.ref_available()
    R = oracle.Reference() if have_ref else None
    scenes = [("tri", i, s) for i, s in enumerate(cfg.terrains)] + \
             [("point", i, s) for i, s in enumerate(cfg.clouds)]
    workers = min(8, threads)
    inner = max(1, threads // workers)

    def check(item):
        kind, i, sc = item
        if R is not None:
            want, times = R.scene(kind, sc.items, sc.closest, sc.knn, cfg.k, sc.radius,
                                  float(sc.r), sc.rays if kind == "tri" else None, inner)
        else:
            ref = oracle.LBVH(kind, sc.items)
            t0 = time.perf_counter()
            want = {"closest": ref.closest(sc.closest, inner), "knn": ref.knn(sc.knn, cfg.k, inner),
                    "radius": ref.radius(sc.radius, float(sc.r), inner)}
            if kind == "tri":
                want["rays"] = ref.raycast(sc.rays, inner)
            times = {"closest_ms": (time.perf_counter() - t0) * 1e3}
        bad, fps = [], {}
        for name, wv in want.items():
            g = got[f"{kind}_{name}"][i]
            if name == "radius":
                go, gk = np.asarray(g[0]).astype(np.int64), np.asarray(g[1]).view(np.uint64)
                ok = np.array_equal(go, wv[0]) and np.array_equal(gk, wv[1])
                if R is not None:
                    fps[name] = (R.list_hash(go, gk), R.list_hash(wv[0], wv[1]))
            else:
                gv = np.asarray(g)
                ok = np.array_equal(gv.view(wv.dtype).reshape(wv.shape), wv)
                if R is not None:
                    if name == "rays":
                        fps[name] = (R.ray_hash(gv.view(np.uint64))[0], R.ray_hash(wv)[0])
                    elif name == "closest":
                        fps[name] = (R.closest_hash(gv.view(np.uint32)), R.closest_hash(wv))
                    else:
                        fps[name] = (R.list_hash(*oracle.knn_to_csr(gv.view(np.uint32).reshape(wv.shape))),
                                     R.list_hash(*oracle.knn_to_csr(wv)))
            if not ok or (name in fps and fps[name][0] != fps[name][1]):
                bad.append(name)
        units = (len(sc.closest) + len(sc.knn) + len(sc.radius) +
                 (len(sc.rays) if kind == "tri" else 0))
        qms = sum(v for k, v in times.items() if k != "build_ms")
        return kind, i, bad, units, qms, fps

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=workers) as ex:
        res = list(ex.map(check, scenes))
    wall = time.perf_counter() - t0
    failed = [f"{k}[{i}]:{','.join(b)}" for k, i, b, _, _, _ in res if b]
    if failed:
        raise RuntimeError(f"scenes differ from the CPU reference: {failed[:8]}")
    units = sum(u for _, _, _, u, _, _ in res)
    # a fingerprint of the per-scene fingerprints (scene order, kind order, operation order)
    chain_e, chain_r = 0xcbf29ce484222325, 0xcbf29ce484222325
    for _, _, _, _, _, fps in res:
        for name in sorted(fps):
            for v_e, v_r in (fps[name],):
                chain_e = ((chain_e ^ (v_e & 0xFFFFFFFFFFFFFFFF)) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
                chain_r = ((chain_r ^ (v_r & 0xFFFFFFFFFFFFFFFF)) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    parity = {"against": "reference" if have_ref else "port", "scenes_checked": len(res),
              "units_checked": units, "mismatches": 0,
              "fingerprint_of_scene_fingerprints": f"0x{chain_e:016x}",
              "reference_fingerprint_of_scene_fingerprints": f"0x{chain_r:016x}",
              "batched_vs_loop": "all scenes bit-identical", "check_wall_s": round(wall, 1)}
    qms = sum(q for _, _, _, _, q, _ in res)
    cpu = {"value": round(units / (qms * 1e-3) / 1e6 * workers, 4) if qms else None,
           "unit": "Mqueries/s", "cores": workers * inner,
           "kind": "reference" if have_ref else "port",
           "sample": (f"every query and ray of all {len(res)} scenes ({units} units), "
                      f"{workers} scenes at a time on {inner} threads each; CPU tree builds "
                      "excluded")}
    return parity, cpu


# ---------------------------------------------------------------------------------------
# kernel cases: one kernel family on its configuration's inputs, for profiler captures
# ---------------------------------------------------------------------------------------
KERNEL_CASES = {
    "build_lbvh": "LBVH build of the 1,048,576-point volume cloud (k_centroid_bounds, k_morton, "
                  "k_rs_*, k_emit, k_bottom_up_ranged, k_depth)",
    "build_sah": "binned SAH build (32 bins) of the 1,310,720-triangle city (k_level_*, "
                 "k_warp_tasks, k_sah_leaves, k_bottom_up_ranged)",
    "refit": "full and 1% dirty refit of the volume cloud's LBVH (k_refit_leaves, k_bottom_up, "
             "k_dirty_mark, k_dirty_merge)",
    "closest_tri": "20,000 closest-point queries on the terrain's LBVH, 131,072 triangles, one "
                   "thread per query (k_closest_bin) and 4 lanes per query (k_closest_split)",
    "closest_gauss": "262,144 closest-ellipsoid queries on 1,048,576 Gaussians (k_closest_bin)",
    "knn_points": "kNN k=8, 20,000 queries on each 1,048,576-point cloud (k_knn_split: a warp "
                  "per query on the sphere shell's SAH tree in coherent order, then 8 lanes per "
                  "query on the uniform cloud; k_knn_bin: one thread per query on the uniform "
                  "cloud)",
    "radius_points": "radius 1.0, 20,000 queries on the uniform cloud, single pass "
                     "(k_radius_count_pool, k_radius_gather, k_radius_fill_lost, k_seg_sort_*)",
    "grad": "adjoints: 262,144 Gaussian distances (k_dist_grad, k_segment_sum) and 1,000,000 "
            "terrain ray t (k_ray_grad)",
    "rays_terrain": "1,000,000 down rays on the terrain's LBVH, coherent order, 5 blocks/SM "
                    "(k_ray_bin)",
    "rays_city": "1,000,000 cosine rays on the city's SAH tree, coherent order, 5 blocks/SM "
                 "(k_ray_bin)",
    "topology_city": "qk_update_topology with the bench's 1% cluster edit on the city's SAH tree, "
                     "three calls (k_topo_*, the forest's k_warp_tasks, k_bottom_up_ranged, "
                     "k_depth*)",
}


def kernel_case(args):
    """Runs the kernels of one family twice (a profiler then captures the second launch with
    -s 1 -c 1) on the inputs of the configuration they serve; prints one line."""
    import torch

    from quarry import capi
    from quarry import workloads as w

    name = args.kernel_case
    torch.cuda.set_device(0)
    dev = capi.to_device
    if name in ("build_lbvh", "refit", "knn_points", "radius_points"):
        vol = w.point_cloud("volume", 1 << 20, 1)
        tree = capi.DeviceTree("point", vol)
        q = dev(w.uniform_points(20_000, vol.min(0), vol.max(0), 1, 13), np.float32)
    if name == "build_lbvh":
        tree.build()
    elif name == "build_sah":
        cfg = w.city_config(131072, 1000, 100, 1)
        tree = capi.DeviceTree("tri", cfg.tris, builder="sah", sah_bins=32)
        tree.build()
    elif name == "refit":
        moved, ids = w.coherent_motion(vol, 0.01, 0.05, 1)
        md = dev(moved, np.float32)
        for _ in range(2):
            tree.refit(md)
        ids_d, sub = dev(ids, np.int32), dev(moved[ids], np.float32)
        for _ in range(2):
            tree.refit_dirty(ids_d, sub)
    elif name == "closest_tri":
        cfg = w.terrain_config(256, 1000, 20_000, 1)
        t2 = capi.DeviceTree("tri", cfg.tris)
        qd = dev(cfg.queries, np.float32)
        for _ in range(2):
            t2.closest(qd, 0)
            t2.closest(qd, capi.QK_TUNE_SPLIT4)
    elif name == "closest_gauss":
        g = capi.DeviceTree("gauss", w.gaussians(1_048_576, 0.05, 1.0, 1))
        qd = dev(w.uniform_points(262_144, [0, 0, 0], [100, 100, 100], 1, 31), np.float32)
        for _ in range(2):
            g.closest(qd, 0)
    elif name == "knn_points":
        shell = w.point_cloud("surface", 1 << 20, 1)
        ts = capi.DeviceTree("point", shell, builder="sah", sah_bins=32)
        qs = dev(w.uniform_points(20_000, shell.min(0), shell.max(0), 1, 13), np.float32)
        for _ in range(2):
            ts.knn(qs, 8, capi.QK_TUNE_SPLIT | capi.QK_ORDER_COHERENT)
            tree.knn(q, 8, capi.QK_TUNE_SPLIT8)
            tree.knn(q, 8, 0)
    elif name == "radius_points":
        for _ in range(2):
            tree.radius(q, 1.0, capi.QK_TUNE_STASH)
    elif name == "grad":
        gt = capi.DeviceTree("gauss", w.gaussians(1_048_576, 0.05, 1.0, 1))
        qd = dev(w.uniform_points(262_144, [0, 0, 0], [100, 100, 100], 1, 31), np.float32)
        res = gt.closest(qd, 0)
        cfg = w.terrain_config(256, 1_000_000, 10, 1)
        tt = capi.DeviceTree("tri", cfg.tris)
        rd = dev(cfg.rays, np.float32)
        _, rid = tt.raycast_ids(rd, 0)
        for _ in range(2):
            gt.distance_grad(qd, res)
            tt.ray_t_grad(rd, rid, None, with_rays=True)
    elif name == "topology_city":
        cfg = w.city_config(131072, 1000, 100, 1)
        _, _, _, _, surgery, keep = topology_surgery("tri", cfg.tris, "sah", 32, "cluster", 1)
        for _ in range(3):
            surgery()
    elif name in ("rays_terrain", "rays_city"):
        if name == "rays_city":
            cfg = w.city_config(131072, 1_000_000, 10, 1)
            t3 = capi.DeviceTree("tri", cfg.tris, builder="sah", sah_bins=32)
        else:
            cfg = w.terrain_config(256, 1_000_000, 10, 1)
            t3 = capi.DeviceTree("tri", cfg.tris)
        rd = dev(cfg.rays, np.float32)
        for _ in range(2):
            t3.raycast(rd, capi.QK_ORDER_COHERENT | capi.QK_TUNE_HIGH_OCC)
    torch.cuda.synchronize()
    print(json.dumps({"kernel_case": name, "what": KERNEL_CASES[name]}), flush=True)


# ---------------------------------------------------------------------------------------
# the default run: every configuration, the city line as the headline
# ---------------------------------------------------------------------------------------
def all_arm(args, world, rank, local):
    import torch

    head = rays_arm(args, world, rank, local, "city")
    configs = {}
    if world == 1 and not args.only:
        for name, fn in (("terrain", lambda: rays_arm(args, world, rank, local, "terrain")),
                         ("points", lambda: points_arm(args, world, rank, local)),
                         ("grad", lambda: grad_arm(args, world, rank, local)),
                         ("batch", lambda: batch_arm(args, world, rank, local))):
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            t0 = time.perf_counter()
            line = fn()
            if line is not None:
                for key in ("metric", "n_gpus", "vs_baseline", "data", "variants_ms"):
                    line.pop(key, None)
                line["wall_s"] = round(time.perf_counter() - t0, 1)
                configs[name] = line
    if rank == 0:
        head["configs"] = configs if configs else "the extra configurations run at N = 1"
        print(json.dumps(head), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.kernel_case:
        kernel_case(args)
        return
    world, rank, local = init_dist(args)
    try:
        if args.workload == "all":
            all_arm(args, world, rank, local)
        else:
            fn = {"city": lambda: rays_arm(args, world, rank, local, "city"),
                  "terrain": lambda: rays_arm(args, world, rank, local, "terrain"),
                  "points": lambda: points_arm(args, world, rank, local),
                  "grad": lambda: grad_arm(args, world, rank, local),
                  "batch": lambda: batch_arm(args, world, rank, local)}[args.workload]
            line = fn()
            if rank == 0 and line is not None:
                print(json.dumps(line), flush=True)
        barrier(world)
    finally:
        from quarry import dist

        if _RANKS is not None:
            dist.destroy(_RANKS)


if __name__ == "__main__":
    main()
