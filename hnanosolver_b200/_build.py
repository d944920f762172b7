"""Compiles libhns.so (the solver's C ABI and its sm_100a kernels) in-tree with nvcc."""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libhns.so")

# -fmad=false: no implicit multiply-add contraction, so that the FP32 kernels round exactly
# as the reference's operations are written (explicit fmaf only where the reference calls
# __fmaf_rn). The kernels are memory-bound; the extra FP instructions cost nothing measurable.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "-shared",
]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def build(verbose: bool = False, extra=()) -> str:
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    cmd = [nvcc, *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-o", LIB, *sources()]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


def build_legacy_test() -> str:
    """The C++ program that drives the reference-named entry points (tests/legacy)."""
    src = os.path.join(ROOT, "tests", "legacy", "legacy_api_test.cpp")
    out_dir = os.path.join(ROOT, "tests", "legacy", "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "legacy_api_test")
    cuda = os.path.dirname(os.path.dirname(os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")))
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"), src,
           "-o", exe, "-L", PKG, "-lhns", "-L", os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN/../../../hnanosolver_b200", "-Wl,-rpath," + os.path.join(cuda, "lib64")]
    subprocess.run(cmd, check=True)
    return exe


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
