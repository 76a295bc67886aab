"""quarry's own callers of gpu/gpu_bvh.h and of the `quarry` module, run against this engine.

The drop-in claim is that code written against quarry's C++ API and Python module works
unchanged.  `oracle/Makefile` (target `callers`, run by the build) compiles quarry's benches
(bench/gpu_bench.cpp, gpu_query_bench.cpp, gpu_cloud_bench.cpp, gpu_gauss_bench.cpp) and
examples (examples/dynamic_scene.cpp, examples/main.cpp) unchanged, against quarry's own
core/ and cpu/ headers and this engine's gpu/gpu_bvh.h, links them with this engine's
libquarry_b200.so and quarry's CPU sources, and byte-compiles quarry's binding test
(python/test_quarry.py).  The binaries check every ray and query against quarry's CPU
reference themselves and exit non-zero on any mismatch (gpu_bench.cpp:381-410,
gpu_query_bench.cpp:767-837); this file runs them on small scenes and requires exit 0.
They also cover the C++ entry points no other test reaches (treeHashGPU,
lastTraversalStatsGPU, lastQueryStatsGPU, warmupQueryGPU, validate*BVHGPU) and print the
per-stage build times (GpuBuildTimings), checked here to be filled.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "oracle" / "_ref" / "bin"
PKG = ROOT / "quarry-gpu_b200"

pytestmark = pytest.mark.gpu


def _run(name: str, *args: str, timeout: int = 600) -> str:
    exe = BIN / name
    if not exe.exists():
        pytest.skip(f"{exe} not built (make -C oracle callers needs quarry's sources)")
    p = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=timeout)
    out = p.stdout + p.stderr
    assert p.returncode == 0, f"{name} {' '.join(args)} exited {p.returncode}:\n{out[-4000:]}"
    assert "FAIL" not in out and "MISMATCH" not in out, out[-4000:]
    return out


def _zero_mismatches(out: str) -> int:
    """Every 'verify ...' line must report zero mismatches of every kind; returns how many
    verify lines were seen."""
    lines = [ln for ln in out.splitlines() if "verify" in ln and "mismatch" in ln]
    for ln in lines:
        for key, val in re.findall(r"(\w*mismatch)=(\d+)", ln):
            assert int(val) == 0, ln
    return len(lines)


def _stage_times(out: str) -> dict:
    m = re.search(r"gpu build morton=([\d.]+) sort=([\d.]+) scatter=([\d.]+) tree=([\d.]+) "
                  r"refit=([\d.]+) total=([\d.]+)", out)
    assert m, out[-2000:]
    return dict(zip(("morton", "sort", "scatter", "tree", "refit", "total"),
                    map(float, m.groups())))


FAST = ("--runs", "2", "--warmup-ms", "20")


@pytest.mark.parametrize("args", [
    ("--grid", "256", "--rays", "200000", "--stats"),
    ("--grid", "128", "--rays", "100000", "--sah", "--stats"),
    ("--grid", "128", "--rays", "100000", "--wide", "--ray-sort"),
    ("--grid", "128", "--rays", "100000", "--ray-sort-dir", "--mode", "random"),
    ("--grid", "128", "--rays", "100000", "--ray-sort-host", "--sah", "--wide"),
    ("--scene", "city", "--buildings", "4096", "--rays", "100000", "--mode", "random", "--sah"),
    ("--scene", "mixed", "--grid", "64", "--random-tris", "20000", "--rays", "50000"),
])
def test_reference_gpu_bench(args):
    out = _run("gpu_bench", *args, *FAST)
    assert "gpu tree PASS" in out
    assert _zero_mismatches(out) == 1
    st = _stage_times(out)
    assert st["total"] > 0 and st["tree"] > 0 and st["refit"] > 0
    if "--sah" not in args:
        assert st["sort"] > 0  # LBVH: Morton / sort stages are timed separately
    else:
        m = re.search(r"gpu sah bin=([\d.]+) split=([\d.]+) partition=([\d.]+)", out)
        assert m and float(m.group(1)) + float(m.group(2)) + float(m.group(3)) > 0
    if "--stats" in args:
        assert re.search(r"avg_node_tests=[1-9]", out) and "stack_overflows=0" in out


@pytest.mark.parametrize("args", [
    ("--query", "closest", "--stats"),
    ("--query", "knn", "--k", "8", "--stats"),
    ("--query", "knn", "--k", "32", "--query-sort"),
    ("--query", "radius", "--radius", "2.0", "--stats"),
    ("--query", "radius", "--radius", "1.0", "--sah", "--query-sort"),
    ("--query", "closest", "--refit", "--refit-motion", "coherent"),
    ("--query", "knn", "--refit", "--sah"),
    ("--query", "closest", "--topo", "--topo-mix", "mixed", "--topo-rounds", "3"),
    ("--query", "knn", "--topo", "--topo-mix", "mixedmid", "--topo-kind", "scatter",
     "--topo-rounds", "3", "--sah"),
    ("--query", "closest", "--topo", "--topo-mix", "delete", "--topo-rounds", "2"),
    ("--query", "closest", "--topo", "--topo-mix", "insertmid", "--topo-rounds", "2"),
    ("--query", "closest", "--topo", "--topo-mix", "move", "--topo-rounds", "2"),
])
def test_reference_gpu_query_bench(args):
    out = _run("gpu_query_bench", "--grid", "128", "--points", "20000", *args, *FAST)
    assert "gpu tree PASS" in out
    assert _zero_mismatches(out) >= 1


@pytest.mark.parametrize("args", [
    ("--kind", "sheet", "--query", "closest", "--stats"),
    ("--kind", "volume", "--query", "knn", "--k", "16", "--wide"),
    ("--kind", "volume", "--query", "radius", "--sah"),
    ("--kind", "sheet", "--query", "knn", "--refit", "--refit-motion", "coherent"),
])
def test_reference_gpu_cloud_bench(args):
    out = _run("gpu_cloud_bench", "--points", "131072", "--queries", "20000", *args, "--runs", "2")
    assert _zero_mismatches(out) >= 1


@pytest.mark.parametrize("args", [
    ("--kind", "sheet", "--query", "closest", "--stats"),
    ("--kind", "volume", "--query", "knn", "--k", "8", "--query-sort", "--wide"),
    ("--kind", "sheet", "--query", "radius", "--sah"),
    ("--kind", "volume", "--query", "closest", "--refit"),
])
def test_reference_gpu_gauss_bench(args):
    out = _run("gpu_gauss_bench", "--gaussians", "65536", "--queries", "10000", *args, "--runs", "2")
    assert _zero_mismatches(out) >= 1


def test_reference_dynamic_scene():
    """80 frames of refits and topology edits on a terrain with moving props, checked against
    quarry's CPU BVH and a fresh build each time; prints treeHashGPU."""
    out = _run("dynamic_scene")
    assert "checks ok" in out
    assert re.search(r"tree hash 0x[0-9a-f]{16}", out)


def test_reference_example():
    out = _run("quarry_example")
    assert "no usable GPU" not in out
    assert "validate: pass" in out and "partial refit" in out


def test_reference_python_binding_test():
    """quarry's python/test_quarry.py, unchanged, importing this engine's `quarry` module."""
    pyc = BIN / "test_quarry.qbc"
    if not pyc.exists():
        pytest.skip(f"{pyc} not built")
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([str(PKG), env.get("PYTHONPATH", "")])
    p = subprocess.run([sys.executable, str(pyc)], capture_output=True, text=True, timeout=900,
                       env=env, cwd=str(ROOT))
    out = p.stdout + p.stderr
    assert p.returncode == 0, out[-4000:]
    assert "PYTHON BINDINGS PASS" in out, out[-4000:]
