"""Build the CUDA library in-tree: kielflow_b200/libkf.so for sm_100a.

Run ``python -m kielflow_b200.build``.  nvcc cross-compiles on a machine
without a GPU; the .so is loaded from the package directory at import time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
SRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libkf.so")
SOURCES = ["kf_capi.cu", "kf_noalloc.cu", "kf_io.cpp"]
HEADERS = ["kf_fft.cuh", "kf_types.cuh", "kf_passes.cuh", "kf_pointwise.cuh", "kf_poisson.cuh", "kf_adjoint.cuh",
           "kf_adjoint_host.cuh", "kf_graph.cuh", "kf_driver.cuh", "kf_io.hpp", "kf_stretch.cuh", "kf_march.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(SRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "kielflow_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [nvcc(), *ARCH, *FLAGS, "-o", LIB + ".tmp", *[os.path.join(SRC, s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
