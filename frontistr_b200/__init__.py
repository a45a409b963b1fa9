"""frontistr_b200: a B200-native (sm_100a) drop-in for FrontISTR's 3x3-block CG solve.

The solver itself is CUDA behind the C ABI of include/hecmw33_gpu.h
(frontistr_b200/lib/libhecmw33_gpu.so); this package is the host-side mirror of
the reference interface (hecmw_solve on a hecmwST_matrix) plus system generators.
"""
from .matrix import HecMatrix, default_iarray_rarray  # noqa: F401

__all__ = ["HecMatrix", "default_iarray_rarray"]
