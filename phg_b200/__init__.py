"""phg_b200: B200 (sm_100a) element assembly + Jacobi-PCG for PHG's
tetrahedral Lagrange P1/P2/P3 path.

The compute path is the CUDA library libphg_b200.so (C ABI in
include/phg_gpu.h, sources in phg_b200/csrc).  This module loads it with
ctypes and offers the same operations with numpy arrays (host memory) or
torch CUDA tensors (device memory).  There is no CPU fallback: if the
library is missing or no GPU is present, calls raise.
"""
from .core import (PhgGpuError, Solver, last_warning, lib, load_library, LIB_PATH)  # noqa: F401
from .mesh import kuhn_cube, lagrange_dofs, sine_source, write_medit  # noqa: F401

__all__ = ["PhgGpuError", "Solver", "last_warning", "lib", "load_library", "LIB_PATH",
           "kuhn_cube", "lagrange_dofs", "sine_source", "write_medit"]
