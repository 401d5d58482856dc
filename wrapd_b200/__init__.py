"""wrapd_b200: WRAPD's ADMM solve loop (georgbrown/wrapd) on one B200.

The numeric path is the CUDA library ``_lib/libwrapd_gpu.so`` (sm_100a) behind
the C ABI of ``include/wrapd_gpu.h``; this package holds its Python binding
(``capi``), a mirror of the reference's ``Solver`` interface (``solver``), the
seeded synthetic bar workloads (``bars``) and the build script (``build``).
"""
from . import bars
from .capi import WrapdError
from .solver import AlgorithmData, Settings, Solver, solve_bar

__all__ = ["bars", "WrapdError", "AlgorithmData", "Settings", "Solver", "solve_bar"]
