"""Schedule autotuner: picks launch shapes and layouts by measuring them, and remembers.

The engine's tunable choices -- block size, persistent blocks per SM, shared-memory
short-stack depth and chunks per fetch of the batched kernels, binary vs 4-wide layout,
Morton ordering, the ray kernel's schedule, the SAH bin count -- never change a result: every
candidate must return the same bits, which the tuner checks through a caller-supplied
fingerprint of the outputs (a candidate that differs is an error, not a slower option).

Search: coordinate descent over the parameter space -- one dimension at a time, the others
held at the best point so far, until a sweep improves nothing (at most `sweeps` sweeps) --
with every point timed as the median of `repeats` CUDA-event measurements after one warm-up
run.  Results persist in a JSON file keyed by device and workload signature, so a second
process with the same workload reuses the choice without measuring.

The cache file is $QUARRY_AUTOTUNE_CACHE, else ~/.cache/quarry_b200/autotune.json.  Choices
measured on B200 for the benchmark workloads ship beside this module (tuned_b200.json) and
are used when the cache has no entry for a key.
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any, Callable

VERSION = 1
SHIPPED = Path(__file__).resolve().parent / "tuned_b200.json"


def default_path() -> Path:
    env = os.environ.get("QUARRY_AUTOTUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "quarry_b200" / "autotune.json"


def cuda_event_timer(run: Callable[[dict], Any], params: dict, repeats: int) -> float:
    """Median device time (ms) of run(params) over `repeats` launches, after one warm-up."""
    import torch

    run(params)
    times = []
    for _ in range(repeats):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run(params)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    times.sort()
    return float(times[len(times) // 2])


class FingerprintMismatch(RuntimeError):
    pass


@dataclass
class Result:
    key: str
    params: dict
    ms: float
    trials: list = field(default_factory=list)
    cached: bool = False
    tuning_s: float = 0.0
    source: str = "measured"


def _canon(params: dict) -> str:
    return json.dumps(params, sort_keys=True)


class Autotuner:
    def __init__(self, path: str | os.PathLike | None = None,
                 timer: Callable[[Callable, dict, int], float] | None = None,
                 device: str | None = None, shipped: str | os.PathLike | None = SHIPPED):
        self.path = Path(path) if path is not None else default_path()
        self.timer = timer or cuda_event_timer
        self.device = device if device is not None else _device_name()
        self.cache = self._load(self.path)
        self.shipped = self._load(Path(shipped)) if shipped is not None else {}

    # ---- persistence ----
    @staticmethod
    def _load(path: Path) -> dict:
        try:
            data = json.loads(path.read_text())
        except (OSError, ValueError):
            return {}
        if not isinstance(data, dict) or data.get("version") != VERSION:
            return {}
        return data.get("entries", {})

    def save(self) -> None:
        self.path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.path.with_suffix(".tmp")
        tmp.write_text(json.dumps({"version": VERSION, "entries": self.cache}, indent=1,
                                  sort_keys=True))
        os.replace(tmp, self.path)

    def full_key(self, key: str) -> str:
        return f"{self.device}|{key}"

    def _entry(self, key: str) -> tuple[dict | None, str]:
        fk = self.full_key(key)
        if fk in self.cache:
            return self.cache[fk], "cache"
        if fk in self.shipped:
            return self.shipped[fk], "shipped"
        return None, ""

    def lookup(self, key: str) -> dict | None:
        e, _ = self._entry(key)
        return None if e is None else dict(e["params"])

    # ---- search ----
    def search(self, key: str, space: dict[str, list], run: Callable[[dict], Any],
               fingerprint: Callable[[dict], Any] | None = None, start: dict | None = None,
               valid: Callable[[dict], bool] | None = None, repeats: int = 3, sweeps: int = 2,
               force: bool = False, tolerance: float = 0.01) -> Result:
        """Best point of `space` for run(); `fingerprint(params)` (called right after a run
        with those params) must be equal for every candidate."""
        fk = self.full_key(key)
        e, src = self._entry(key)
        if not force and e is not None:
            return Result(key, dict(e["params"]), float(e["ms"]), list(e.get("trials", [])),
                          cached=True, source=src)
        t0 = time.perf_counter()
        valid = valid or (lambda p: True)
        cur = dict(start) if start is not None else {k: v[0] for k, v in space.items()}
        if not valid(cur):
            raise ValueError(f"start point {cur} is not valid")
        seen: dict[str, float] = {}
        trials = []
        ref_fp = [None]

        def measure(p: dict) -> float:
            c = _canon(p)
            if c in seen:
                return seen[c]
            ms = self.timer(run, p, repeats)
            if fingerprint is not None:
                fp = fingerprint(p)
                if ref_fp[0] is None:
                    ref_fp[0] = fp
                elif fp != ref_fp[0]:
                    raise FingerprintMismatch(f"{key}: {p} changed the results")
            seen[c] = ms
            trials.append({"params": dict(p), "ms": round(ms, 4)})
            return ms

        best = measure(cur)
        for _ in range(max(1, sweeps)):
            improved = False
            for dim, values in space.items():
                for v in values:
                    if v == cur[dim]:
                        continue
                    cand = dict(cur)
                    cand[dim] = v
                    if not valid(cand):
                        continue
                    ms = measure(cand)
                    if ms < best * (1.0 - tolerance):
                        cur, best, improved = cand, ms, True
            if not improved:
                break
        res = Result(key, cur, best, trials, cached=False, tuning_s=time.perf_counter() - t0)
        self.cache[fk] = {"params": cur, "ms": best, "trials": trials}
        return res


def _device_name() -> str:
    try:
        from . import capi

        return capi.describe() or "no-device"
    except Exception:
        return "no-device"


# ---------------------------------------------------------------------------------------
# the engine's spaces
# ---------------------------------------------------------------------------------------
BATCH_SPACE = {
    # QK_ORDER_MORTON = 1, QK_WIDE = 4; QK_TUNE_STASH = 8192 (single-pass radius, radius only)
    "flags": [0, 1, 4, 5, 8192, 8193, 8196, 8197],
    "block": [128, 64, 256],
    "blocks_per_sm": [6, 4, 8, 2],
    "short_stack": [8, 0, 16],
    "chunks_per_fetch": [1, 4, 16],
    "split": [0, 1],                       # one warp per query (closest / kNN / radius)
}

BATCH_START = {"flags": 1, "block": 128, "blocks_per_sm": 6, "short_stack": 8,
               "chunks_per_fetch": 1, "split": 0}


def batch_launch(params: dict) -> dict:
    """The qk_batch_tune fields of a batch point."""
    out = {k: params[k] for k in ("block", "blocks_per_sm", "short_stack", "chunks_per_fetch")}
    out["split"] = params.get("split", 0)
    return out


def batch_valid(op: str):
    """Points of BATCH_SPACE an operation accepts: the split schedule serves closest, kNN and
    radius on binary nodes; the single-pass flag is for radius plans (and the thread-per-query
    schedule)."""
    def ok(p: dict) -> bool:
        if p["flags"] & 8192 and (op != "radius" or p.get("split", 0)):
            return False
        if not p.get("split", 0):
            return True
        return op != "rays" and not (p["flags"] & 4)
    return ok


RAY_SPACE = {
    "builder": ["sah32", "lbvh", "sah16", "sah8"],
    "layout": ["bin", "wide"],
    "order": ["input", "morton"],
    "schedule": ["occ", "plain", "dyn", "dyn_occ", "sm", "occ_sm", "leaf4", "occ_leaf4"],
}


def ray_valid(p: dict) -> bool:
    # the schedule variants exist for the binary kernel only
    return p["layout"] == "bin" or p["schedule"] == "plain"


def ray_flags(p: dict) -> int:
    from . import capi

    f = capi.QK_WIDE if p["layout"] == "wide" else 0
    if p["order"] == "morton":
        f |= capi.QK_ORDER_MORTON
    if p["layout"] == "bin":
        f |= {"plain": 0, "occ": capi.QK_TUNE_HIGH_OCC, "dyn": capi.QK_TUNE_DYNAMIC,
              "dyn_occ": capi.QK_TUNE_DYNAMIC | capi.QK_TUNE_HIGH_OCC,
              "sm": capi.QK_TUNE_SHORT_STACK,
              "occ_sm": capi.QK_TUNE_HIGH_OCC | capi.QK_TUNE_SHORT_STACK,
              "leaf4": capi.QK_TUNE_LEAF4,
              "occ_leaf4": capi.QK_TUNE_HIGH_OCC | capi.QK_TUNE_LEAF4}[p["schedule"]]
    return f
