"""B200-native MCSA (Monte Carlo Synthetic Acceleration) for MCLS.

The product is libmclsgpu.so (C ABI: include/mclsgpu.h; C++ facade with the
reference's class names: include/MCLS_*.hpp).  This package holds its CUDA
sources (csrc/), the in-tree build (build.py), a ctypes binding of the C ABI
(capi.py) and the seeded synthetic workloads (problems.py).
"""
from . import problems  # noqa: F401

__all__ = ["problems", "capi", "build"]
