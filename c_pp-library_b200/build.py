"""Builds libawcm_b200.so in-tree: the CUDA kernels and the C-ABI for sm_100a.

    python c_pp-library_b200/build.py [--force]

Flags: -gencode arch=compute_100a,code=sm_100a, -O3, -lineinfo, --fmad=false (the reference's
IEEE double arithmetic has no fused multiply-add; keeping products and sums separately rounded is
what makes results bit-identical to it).  The adjoint kernels (awcm2d_adjoint.cu) are a derivative
checked against finite differences rather than a bit-exact restatement, and build with
--fmad=true.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libawcm_b200.so")
SOURCES = ["awcm_common.cu", "awcm2d.cu", "awcm1d.cu", "awcm2d_adjoint.cu", "awcm_state.cpp"]
HEADERS = ["awcm_common.cuh", "awcm_numerics.cuh", "awcm2d_types.cuh"]
# per-file overrides of the contraction flags
FMA_SOURCES = {"awcm2d_adjoint.cu"}

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "awcm_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        flags = NVCC_FLAGS
        if src in FMA_SOURCES:
            flags = [f.replace("--fmad=false", "--fmad=true").replace("-ffp-contract=off", "-ffp-contract=fast")
                     for f in NVCC_FLAGS]
        cmd = [_nvcc(), *flags, "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
