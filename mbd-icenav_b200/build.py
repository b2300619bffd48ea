"""Build ``libdem_b200.so`` (the C-ABI library) for sm_100a with nvcc.

The library is built in-tree next to this file so that it travels with the
repository snapshot.  ``-fmad=false`` keeps every multiply-add rounded twice,
as NumPy and XLA-CPU compute them, so that contact and fracture predicates
evaluated from identical inputs agree bit for bit with the oracle.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB_NAME = "libdem_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)

SOURCES = [os.path.join(CSRC, f) for f in ("dem_b200.cu", "dem_costmap.cu", "dem_rollout.cu", "sg_kernels.cu")]
DEPS = SOURCES + [os.path.join(CSRC, f) for f in ("dem_kernels.cuh", "dem_math.cuh", "sg_tc.cuh")] + [
    os.path.join(INCLUDE, f) for f in ("dem_b200.h", "surrogate_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-O2", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libdem_b200.so")
    return cand


def needs_build(path: str = LIB_PATH) -> bool:
    if not os.path.exists(path):
        return True
    t = os.path.getmtime(path)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build_library(force: bool = False, verbose: bool = False, extra_flags=None, out: str = LIB_PATH) -> str:
    """Compile the library if any source is newer than it; return its path."""
    if not force and not needs_build(out):
        return out
    cmd = [nvcc_path(), *NVCC_FLAGS, *(extra_flags or []), "-I", INCLUDE, "-I", CSRC,
           "-o", out + ".tmp", *SOURCES, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libdem_b200.so")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True,
                  extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
