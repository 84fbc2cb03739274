"""Build libmfgpu.so in-tree for sm_100a (B200).

    python pureumfpack.jl_b200/build.py [--verbose]

Compiles the CUDA kernels, the C ABI and the host-side symbolic analysis into
one shared library next to the Python package (pureumfpack/libmfgpu.so).  No
GPU is needed: nvcc cross-compiles.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "pureumfpack", "libmfgpu.so")
SOURCES = [
    "csrc/mfgpu.cu",
    "csrc/costmodel.cu",
    "csrc/gplu.cu",
    "csrc/plan.cpp",
    "csrc/host/symbolic.cpp",
    "csrc/host/api_host.cpp",
]
DEPENDS = SOURCES + [
    "csrc/plan.h",
    "csrc/host/symbolic.h",
    "csrc/device/common.cuh",
    "csrc/device/factor_kernels.cuh",
    "csrc/device/gemm_kernels.cuh",
    "csrc/device/solve_kernels.cuh",
    "csrc/device/tc_gemm.cuh",
    "csrc/device/solve_persistent.cuh",
    "csrc/device/gplu_kernels.cuh",
    "../include/mfgpu.h",
]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-Wall",
    "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(os.path.join(HERE, s)) <= t for s in DEPENDS)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-o", OUT, *[os.path.join(HERE, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=HERE)
    return OUT


if __name__ == "__main__":
    verbose = "--verbose" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=True, verbose=verbose, extra=extra))
