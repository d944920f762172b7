"""B200-native sparse smoke/fire solver on leaf-dense NanoVDB index grids.

The product is libhns.so: hand-written sm_100a CUDA kernels behind the C ABI in
include/hns.h (and the C++ surface in include/hns_legacy.hpp). This package holds its
sources (csrc/), its in-tree build (_build.py), a ctypes binding (lib.py) and the seeded
synthetic workloads (synth.py).
"""
__all__ = ["lib", "synth"]
