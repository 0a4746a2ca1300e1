"""dsem_b200: B200-native (sm_100a, FP64) right-hand side and low-storage
Runge-Kutta stage of the DSEM compressible Navier-Stokes solver.

The compute path is libdsem_b200.so (CUDA kernels behind the C-ABI of
include/dsem_gpu.h); `solver.Solver` is its ctypes front end and `mesh`
builds mesh descriptors for standalone runs.
"""
from . import mesh  # noqa: F401

__all__ = ["mesh", "solver"]
