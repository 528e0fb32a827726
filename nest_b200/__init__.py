"""nest_b200: B200-native implementation of nest's Euler hot path.

The compute path is the CUDA library nest_b200/lib/libnest_b200.so (C ABI in
include/nest_b200.h).  Importing this package loads it; there is no CPU
fallback.
"""
from ._capi import (BC_OUTFLOW, BC_PERIODIC, F32, F64, FLAG_FP32_SCALAR, FLAG_LIMITER_MC, FLAG_LIMITER_NONE,
                    FLAG_NO_RESIDENT, FLAG_REPAIR, FLAG_SPLIT_COMPAT,
                    FLAG_TOTALS, LAYOUT_EXTENDED, LAYOUT_INTERIOR, LIB_PATH, NestError)
from .batch import Batch
from .exchange import PeriodicExchange
from .pipeline import Pipeline, sod1d_pipeline
from .solver import Euler1DGPU, Solver

__all__ = [
    "Batch", "PeriodicExchange", "Pipeline", "sod1d_pipeline", "Euler1DGPU", "Solver", "NestError", "BC_PERIODIC", "BC_OUTFLOW", "F64", "F32",
    "LAYOUT_EXTENDED", "LAYOUT_INTERIOR", "FLAG_TOTALS", "FLAG_REPAIR", "FLAG_NO_RESIDENT", "FLAG_FP32_SCALAR", "FLAG_SPLIT_COMPAT",
    "FLAG_LIMITER_MC", "FLAG_LIMITER_NONE",
    "LIB_PATH",
]
