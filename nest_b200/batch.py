"""Batched independent 2D problems (see nest_batch_* in include/nest_b200.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from ._capi import check, lib

_vp, _i, _d = C.c_void_p, C.c_int, C.c_double


class BatchDesc(C.Structure):
    _fields_ = [("count", C.c_int), ("nx", C.POINTER(C.c_int)), ("ny", C.POINTER(C.c_int)),
                ("dx", C.POINTER(C.c_double)), ("dy", C.POINTER(C.c_double)), ("gamma", C.c_double),
                ("bc_x", C.c_int), ("bc_y", C.c_int), ("precision", C.c_int), ("flags", C.c_int),
                ("stream", C.c_void_p)]


A.bind({
    "nest_batch_create": (_i, [C.POINTER(BatchDesc), C.POINTER(_vp)]),
    "nest_batch_destroy": (_i, [_vp]),
    "nest_batch_upload": (_i, [_vp, _i, _vp, _i]),
    "nest_batch_download": (_i, [_vp, _i, _vp, _i]),
    "nest_batch_step": (_i, [_vp, _i, _d]),
    "nest_batch_step_profiled": (_i, [_vp, _i, _d, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "nest_batch_times": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "nest_batch_totals": (_i, [_vp, C.POINTER(C.c_double)]),
    "nest_batch_set_tiling": (_i, [_vp, _i, _i, _i]),
    "nest_batch_info": (_i, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "nest_batch_reset": (_i, [_vp]),
})


class Batch:
    def __init__(self, nx, ny, gamma=1.4, bc=(A.BC_PERIODIC, A.BC_PERIODIC), precision=A.F32, flags=0,
                 stream=None, dx=None, dy=None):
        if isinstance(bc, int):
            bc = (bc, bc)
        self.nx = np.ascontiguousarray(nx, dtype=np.int32)
        self.ny = np.ascontiguousarray(ny, dtype=np.int32)
        self.count = len(self.nx)
        self.dtype = np.float64 if precision == A.F64 else np.float32
        self._dx = None if dx is None else np.ascontiguousarray(dx, dtype=np.float64)
        self._dy = None if dy is None else np.ascontiguousarray(dy, dtype=np.float64)
        dp = C.POINTER(C.c_double)
        d = BatchDesc(self.count, self.nx.ctypes.data_as(C.POINTER(C.c_int)), self.ny.ctypes.data_as(C.POINTER(C.c_int)),
                      self._dx.ctypes.data_as(dp) if self._dx is not None else None,
                      self._dy.ctypes.data_as(dp) if self._dy is not None else None,
                      gamma, bc[0], bc[1], precision, flags, C.c_void_p(stream) if stream else None)
        h = C.c_void_p()
        check(lib.nest_batch_create(C.byref(d), C.byref(h)), "nest_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.nest_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def upload(self, p: int, U: np.ndarray, layout: int = A.LAYOUT_EXTENDED):
        U = np.ascontiguousarray(U, dtype=self.dtype)
        check(lib.nest_batch_upload(self._h, p, U.ctypes.data, layout), "nest_batch_upload")

    def download(self, p: int, layout: int = A.LAYOUT_EXTENDED) -> np.ndarray:
        g = 4 if layout == A.LAYOUT_EXTENDED else 0
        U = np.zeros((4, int(self.nx[p]) + g, int(self.ny[p]) + g), dtype=self.dtype)
        check(lib.nest_batch_download(self._h, p, U.ctypes.data, layout), "nest_batch_download")
        return U

    def step(self, nsteps: int, cfl: float):
        check(lib.nest_batch_step(self._h, nsteps, cfl), "nest_batch_step")

    def step_profiled(self, nsteps: int, cfl: float):
        ms = np.zeros(2 * nsteps, dtype=np.float32)
        tot = C.c_float(0)
        check(lib.nest_batch_step_profiled(self._h, nsteps, cfl, ms.ctypes.data_as(C.POINTER(C.c_float)),
                                           C.byref(tot)), "nest_batch_step_profiled")
        return ms[0::2].astype(np.float64), ms[1::2].astype(np.float64), float(tot.value)

    def times(self):
        t = np.zeros(self.count)
        s = np.zeros(self.count, dtype=np.int32)
        check(lib.nest_batch_times(self._h, t.ctypes.data_as(C.POINTER(C.c_double)),
                                   s.ctypes.data_as(C.POINTER(C.c_int))), "nest_batch_times")
        return t, s

    def totals(self):
        out = np.zeros((self.count, 4))
        check(lib.nest_batch_totals(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "nest_batch_totals")
        return out

    def set_tiling(self, rows_per_tile: int, warps_per_block: int, blocks_per_sm: int = 0):
        check(lib.nest_batch_set_tiling(self._h, rows_per_tile, warps_per_block, blocks_per_sm),
              "nest_batch_set_tiling")

    def reset(self):
        check(lib.nest_batch_reset(self._h), "nest_batch_reset")

    def info(self):
        c, it, bl = C.c_longlong(), C.c_int(), C.c_int()
        check(lib.nest_batch_info(self._h, C.byref(c), C.byref(it), C.byref(bl)), "nest_batch_info")
        return c.value, it.value, bl.value
