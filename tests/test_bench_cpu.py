"""bench.py's host-side pieces, without a GPU: the reference arm's JSON line (it times
quarry's CPU code on the host) and the host recomputation of the coherent ray order that
the roofline measurement uses."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--small",
                          "--steps", "1", "--warmup", "1"], cwd=ROOT, capture_output=True,
                         text=True, timeout=600, check=True)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:
        return
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["unit"] == "Mrays/s" and line["higher_is_better"] is True
    assert line["config"]["workload"] == "city"
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] >= 1 and cb["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_coherent_order_is_a_grouping_permutation():
    sys.path.insert(0, str(ROOT))
    import bench
    from quarry import workloads

    rays = workloads.cosine_rays(50_000, 0.0, 500.0, 0.0, 400.0, 80.0, 3)
    perm = bench.coherent_order(rays)
    assert np.array_equal(np.sort(perm), np.arange(len(rays)))
    # neighbours in the order start closer together than neighbours in input order
    o = rays[:, :2]
    step_sorted = np.linalg.norm(np.diff(o[perm], axis=0), axis=1).mean()
    step_input = np.linalg.norm(np.diff(o, axis=0), axis=1).mean()
    assert step_sorted < 0.5 * step_input
    # flat input (every ray equal) keeps input order
    same = np.repeat(rays[:1], 100, axis=0)
    assert np.array_equal(bench.coherent_order(same), np.arange(100))


def test_reference_arm_loads_only_checker_libraries_and_matches_the_config():
    """The CPU arm must not load any library of the engine (its inputs come from the
    stand-alone generator build under oracle/_build), and its `config` must be the engine
    arm's (both come from bench.make_workload)."""
    code = (
        "import sys, json\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--small', '--steps', '1', '--warmup', '1']\n"
        "sys.path.insert(0, '.')\n"
        "import bench\n"
        "bench.main()\n"
        "maps = open('/proc/self/maps').read().splitlines()\n"
        "libs = sorted({l.split()[-1] for l in maps if l.split()[-1].endswith('.so')})\n"
        "print(json.dumps({'libs': libs, 'mods': [m for m in sys.modules if m.startswith('quarry')]}))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=600, check=True)
    lines = out.stdout.strip().splitlines()
    line, loaded = json.loads(lines[-2]), json.loads(lines[-1])
    ours = [p for p in loaded["libs"] if str(ROOT) in p]
    assert ours and all("/oracle/" in p for p in ours), ours
    assert loaded["mods"] == []
    sys.path.insert(0, str(ROOT))
    import bench
    import oracle

    assert line["config"] == bench.make_workload(oracle.standalone_workloads(), "city", True, 0)[1]
