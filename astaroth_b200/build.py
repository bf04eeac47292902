"""Builds libastaroth_b200.so in-tree with nvcc for sm_100a (and the C sample).

Run as ``python -m astaroth_b200.build`` or call :func:`build`.  Objects go
to ``astaroth_b200/_build/``; the shared library is written next to this file
so that it travels with the source tree.  Rebuilds only what changed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libastaroth_b200.so"
SAMPLE = PKG / "ac_devicetest"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-Xptxas", "-warn-spills",
    f"-I{INCLUDE}", f"-I{CSRC}",
]
CC_FLAGS = ["-O2", "-fPIC", "-fopenmp", "-std=c11", "-Wall", f"-I{INCLUDE}"]

CU_SOURCES = ["device.cu", "device_data.cu", "device_adjoint.cu", "solve.cu", "solve_tiled.cu",
              "boundconds.cu", "reduce.cu", "cfl.cu", "adjoint.cu", "ensemble.cu", "forcing.cu",
              "bfield.cu", "energy.cu"]
C_SOURCES = ["host.c"]
HEADERS = ["internal.h", "mhd_rhs.cuh", "mhd_rhs_adjoint.cuh", "stencil_plain.cuh", "solve_cell.cuh",
           "halo.cuh", "tma_ring.cuh", "tmem.cuh", "device_impl.h"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compiles every CUDA source for sm_100a and links the shared library."""
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "astaroth_b200.h"]
    objects = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        if force or _stale(o, [s] + headers):
            _run([nvcc, *NVCC_FLAGS, "-c", str(s), "-o", str(o)], verbose)
        objects.append(o)
    for src in C_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".c.o")
        if force or _stale(o, [s, INCLUDE / "astaroth_b200.h"]):
            _run(["gcc", *CC_FLAGS, "-c", str(s), "-o", str(o)], verbose)
        objects.append(o)
    if force or _stale(LIB, objects):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objects),
              "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    sample_src = CSRC / "ac_devicetest.c"
    if sample_src.exists() and (force or _stale(SAMPLE, [sample_src, LIB])):
        _run(["gcc", "-O2", "-std=c11", f"-I{INCLUDE}", str(sample_src), "-o", str(SAMPLE),
              f"-L{PKG}", "-lastaroth_b200", "-Wl,-rpath,$ORIGIN", "-lm"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
