"""Builds libcmf_b200.so in-tree (sm_100a device code + the host model core) and libcmf_synth.so
(host loops of the synthetic-case generator).

    python cama-flood_v4_b200/build.py            # build if sources changed
    python cama-flood_v4_b200/build.py --force

Device code is compiled with -fmad=false: the physics must not fuse multiplies and adds, so
every FP64 operation rounds exactly where the reference's does.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libcmf_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["cmf_engine.cu", "cmf_emu.cu", "cmf_host.cpp"]
HEADERS = ["cmf_kernels.cuh"]
SYNTH_LIB = os.path.join(LIBDIR, "libcmf_synth.so")
SYNTH_SOURCE = "cmf_synth.cpp"
# the generator's loops must round like numpy's element-wise operations: no contraction
SYNTH_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fno-fast-math",
    "-shared", "-cudart", "shared",
]


def _nvcc() -> str:
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.exists(c) or c == "nvcc":
            return c
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "cmf_gpu.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build_synth(force: bool = False, verbose: bool = False) -> str:
    src = os.path.join(CSRC, SYNTH_SOURCE)
    deps = [src, __file__]
    if not force and os.path.exists(SYNTH_LIB) and all(os.path.getmtime(d) <= os.path.getmtime(SYNTH_LIB) for d in deps):
        return SYNTH_LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = ["g++", *SYNTH_FLAGS, "-o", SYNTH_LIB, src]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return SYNTH_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    build_synth(force, verbose)
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-o", LIB] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
