"""B200-native (sm_100a) re-implementation of StarHub's per-frame warp-field solve.

The product is libwarpsolve.so (C ABI: include/warpsolve.h).  This package
holds its build script, a ctypes binding, a host-side mirror of the
reference's WarpSolver interface, the batched / served front ends and the
synthetic scene generator used by the tests and the benchmark.
"""
from ._lib import WarpSolveError, WS_PREC_FP32, WS_PREC_MIXED  # noqa: F401

__all__ = ["WarpSolveError", "WS_PREC_FP32", "WS_PREC_MIXED"]
