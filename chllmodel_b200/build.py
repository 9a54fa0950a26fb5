"""Builds libchll_mod.so (the sm_100a CUDA library) in-tree with nvcc.

Usage: ``python -m chllmodel_b200.build``.  The shared library lands next to
this file so it travels with the source tree; nothing is installed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libchll_mod.so")
SOURCES = ["sweep.cu", "batched.cu", "pooled.cu", "resident.cu", "layout.cu", "observables.cu",
           "adjoint.cu", "analysis.cu", "capi.cu", "noalloc.cu"]
HEADERS = ["chll_common.cuh", "chll_physics.cuh", "sweep.cuh", "sweep_unit.cuh", "moments.cuh",
           "staged.cuh", "pooled.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libchll_mod.so")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "chll_mod.h"))
    return any(os.path.exists(p) and os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every .cu source into one shared library for sm_100a."""
    if not force and not _stale():
        return LIB
    srcs = [os.path.join(CSRC, f) for f in SOURCES if os.path.exists(os.path.join(CSRC, f))]
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", "-o", tmp, *srcs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
