"""ctypes binding of libnest_b200.so (the C ABI declared in include/nest_b200.h).

The library is the product: importing this module loads it and raises
ImportError when it has not been built.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("NEST_B200_LIB", PKG / "lib" / "libnest_b200.so"))

NEST_OK = 0
NEST_ERR_INVALID = 1
NEST_ERR_CUDA = 2
NEST_ERR_OOM = 3
NEST_ERR_NUMERIC = 4
NEST_ERR_UNSUPPORTED = 6
STATUS_NAMES = {
    0: "NEST_OK", 1: "NEST_ERR_INVALID", 2: "NEST_ERR_CUDA", 3: "NEST_ERR_OOM",
    4: "NEST_ERR_NUMERIC", 6: "NEST_ERR_UNSUPPORTED",
}
BC_PERIODIC, BC_OUTFLOW = 0, 1
F64, F32 = 0, 1
LAYOUT_EXTENDED, LAYOUT_INTERIOR = 0, 1
FLAG_TOTALS, FLAG_REPAIR, FLAG_NO_RESIDENT, FLAG_FP32_SCALAR, FLAG_SPLIT_COMPAT = 1, 2, 4, 8, 16
FLAG_LIMITER_MC, FLAG_LIMITER_NONE = 32, 64


class NestError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class SolverDesc(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("halo", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("gamma", C.c_double),
        ("bc_x", C.c_int), ("bc_y", C.c_int), ("precision", C.c_int), ("flags", C.c_int),
        ("stream", C.c_void_p),
    ]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is not built: run `python nest_b200/build.py` (needs nvcc for sm_100a)")
    return C.CDLL(str(LIB_PATH))


lib = _load()

_vp, _dp, _ip, _i, _d = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.c_double
_SIGS = {
    "nest_last_error": (C.c_char_p, []),
    "nest_version": (_i, []),
    "euler1d_gpu_create": (_vp, [_i, _i, _d, _d]),
    "euler1d_gpu_destroy": (None, [_vp]),
    "euler1d_gpu_upload": (None, [_vp, _dp]),
    "euler1d_gpu_download": (None, [_vp, _dp]),
    "euler1d_gpu_compute_dt": (_d, [_vp, _d]),
    "euler1d_gpu_rk2_step": (None, [_vp, _d]),
    "euler1d_gpu_run": (_i, [_vp, _d, _d]),
    "euler1d_gpu_run_timed": (_d, [_vp, _d, _d, _ip]),
    "euler1d_gpu_set_bc": (_i, [_vp, _i]),
    "euler1d_gpu_status": (_i, [_vp]),
    "nest_solver_create": (_i, [C.POINTER(SolverDesc), C.POINTER(_vp)]),
    "nest_solver_destroy": (_i, [_vp]),
    "nest_solver_upload": (_i, [_vp, _vp, _i]),
    "nest_solver_download": (_i, [_vp, _vp, _i]),
    "nest_solver_upload_device": (_i, [_vp, _vp, _i]),
    "nest_solver_download_device": (_i, [_vp, _vp, _i]),
    "nest_solver_step": (_i, [_vp, _i, _d]),
    "nest_solver_step_dt": (_i, [_vp, _i, _d]),
    "nest_solver_step_profiled": (_i, [_vp, _i, _d, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "nest_solver_run_to": (_i, [_vp, _d, _d, _i, _ip]),
    "nest_solver_compute_dt": (_i, [_vp, _d, _dp]),
    "nest_solver_time": (_i, [_vp, _dp, _ip]),
    "nest_solver_reset_time": (_i, [_vp]),
    "nest_solver_totals": (_i, [_vp, _dp]),
    "nest_solver_repairs": (_i, [_vp, C.POINTER(C.c_uint)]),
    "nest_solver_sync": (_i, [_vp]),
    "nest_solver_set_tiling": (_i, [_vp, _i, _i]),
    "nest_solver_set_dt_sequence": (_i, [_vp, _dp, _i, _i]),
    "nest_solver_get_dts": (_i, [_vp, _dp, _i]),
    "nest_solver_state_ptr": (_i, [_vp, C.POINTER(_vp), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "nest_solver_set_exchange_sides": (_i, [_vp, _i, _i]),
    "nest_solver_stage": (_i, [_vp, _i, _d, _d]),
    "nest_solver_speed_slot": (_i, [_vp, C.POINTER(_vp)]),
    "nest_solver_stage_ptr": (_i, [_vp, C.POINTER(_vp)]),
    "nest_solver_stream": (_i, [_vp, C.POINTER(_vp)]),
    "nest_solver_set_time": (_i, [_vp, _d, _i]),
    "nest_write_dat_1d": (_i, [C.c_char_p, _vp, _i, _i, _i, _d, _d, _d, _d]),
    "nest_write_dat_2d": (_i, [C.c_char_p, _vp, _i, _i, _i, _i, _d, _d, _d, _d, _d, _d, _i]),
    "nest_solver_write_dat": (_i, [_vp, C.c_char_p, _i, _i, _d, _d, _d, _d, _i]),
    "nest_solver_save": (_i, [_vp, C.c_char_p]),
    "nest_solver_load": (_i, [_vp, C.c_char_p]),
    "nest_euler1d_run_noalloc": (_i, [_vp, _i, _i, _d, _d, _i, _d, _d, _ip, _dp, _vp]),
}
NOALLOC_MAX_CELLS = 65552


def bind(sigs: dict) -> None:
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


bind(_SIGS)


def last_error() -> str:
    m = lib.nest_last_error()
    return m.decode() if m else ""


def check(status: int, where: str) -> None:
    if status != NEST_OK:
        raise NestError(status, where, last_error())
