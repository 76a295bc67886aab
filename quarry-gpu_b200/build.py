"""Build recipe of the B200 engine: nvcc for the CUDA sources (sm_100a only), gcc for the
workload generators, one shared library with the C ABI, plus the pybind11 module `quarry`.

    python quarry-gpu_b200/build.py            # incremental
    python quarry-gpu_b200/build.py --force    # rebuild everything

Outputs (git-ignored, shipped with the source tree):
    quarry-gpu_b200/quarry/libquarry_b200.so
    quarry-gpu_b200/quarry/_quarry.<ext-suffix>
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import sysconfig
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "quarry"
OBJ = PKG / "_build"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_INC = "/usr/local/cuda/include"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills",
]
CU_SOURCES = ["qk_sort.cu", "qk_build.cu", "qk_sah.cu", "qk_query.cu", "qk_grad.cu",
              "qk_capi.cu", "qk_noalloc.cu", "qk_batch.cu", "qk_topo.cu", "gpu_bvh.cu"]
C_SOURCES = ["scenes.c"]
LIB = OUT / "libquarry_b200.so"


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + \
        sorted((ROOT / "include").rglob("*.h"))


def build(force: bool = False, python_module: bool = True) -> Path:
    OBJ.mkdir(exist_ok=True)
    objs = []
    hdrs = headers()
    for src in CU_SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = OBJ / (s.stem + ".o")
        if force or _stale(o, [s] + hdrs):
            _run([NVCC, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-c", str(s), "-o", str(o)])
        objs.append(o)
    for src in C_SOURCES:
        s = CSRC / src
        o = OBJ / (s.stem + ".o")
        if force or _stale(o, [s] + hdrs):
            _run(["gcc", "-O2", "-fPIC", "-std=c11", "-ffp-contract=off", "-fno-fast-math",
                  "-Wall", "-c", str(s), "-o", str(o)])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(LIB),
              *map(str, objs), "-lm"])
    if python_module:
        build_python(force)
    return LIB


def build_python(force: bool = False) -> Path | None:
    src = CSRC / "quarry_py.cpp"
    if not src.exists():
        return None
    import pybind11

    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    target = OUT / f"_quarry{suffix}"
    if force or _stale(target, [src, LIB] + headers()):
        inc = sysconfig.get_paths()["include"]
        _run(["g++", "-O2", "-shared", "-fPIC", "-std=c++17", "-fvisibility=hidden",
              "-I", pybind11.get_include(), "-I", inc, "-I", str(ROOT / "include"),
              "-I", CUDA_INC, str(src), "-o", str(target), "-L", str(OUT), "-lquarry_b200",
              "-Wl,-rpath,$ORIGIN"])
    return target


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-python", action="store_true")
    a = ap.parse_args()
    build(a.force, not a.no_python)
    sys.exit(0)
