"""Build recipe for the native engine library (liboems_b200.so).

Compiles the CUDA sources under csrc/ for sm_100a with nvcc into a shared
library that sits next to this file, so it travels with the repository.  The
library links the CUDA runtime statically and has no PyTorch dependency: its
only interface is the C ABI in include/oems.h.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liboems_b200.so")
SOURCES = ["csrc/engine.cu", "csrc/host.cpp", "csrc/noalloc.cu", "csrc/sweep.cpp", "csrc/predictor_kernels.cu",
           "csrc/cylindrical.cu"]
HEADERS = ["csrc/yee_kernels.cuh", "csrc/yee_pipe.cuh", "csrc/yee_tma.cuh", "csrc/mur.cuh", "csrc/lumped_ade.cuh",
           "csrc/fd_nf2ff.cuh", "csrc/upml.cuh", "csrc/interface.cuh", "csrc/gemm_tc.cuh", "../include/oems.h",
           "../include/oems_host.h", "../include/oems_predictor.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2,-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-shared",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(HERE, s) for s in SOURCES + HEADERS] + [os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra_flags=()) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, *extra_flags, "-I", os.path.join(ROOT, "include"),
           *[os.path.join(HERE, s) for s in SOURCES], "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
