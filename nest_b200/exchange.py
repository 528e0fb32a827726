"""Patch halo exchange on nest's per-patch storage (nest_exchange_* in
include/nest_b200.h): the device counterpart of nest's
build_periodic_mesh_1d/2d + execute_all_exchanges (include/nest/patch.hpp)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from ._capi import check, lib

_vp, _i = C.c_void_p, C.c_int
A.bind({
    "nest_exchange_create_periodic": (_i, [_i, _i, _i, _i, _i, _i, _i, C.POINTER(_vp)]),
    "nest_exchange_destroy": (_i, [_vp]),
    "nest_exchange_layout": (_i, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "nest_exchange_execute": (_i, [_vp, _vp, _i, _vp]),
})


class PeriodicExchange:
    def __init__(self, dim: int, nx: int, npx: int, nvars: int, halo: int, ny: int = 1, npy: int = 1):
        self.dim, self.nvars, self.halo = dim, nvars, halo
        self.npatch = npx * (npy if dim == 2 else 1)
        h = C.c_void_p()
        check(lib.nest_exchange_create_periodic(dim, nx, ny, npx, npy, nvars, halo, C.byref(h)),
              "nest_exchange_create_periodic")
        self._h = h
        self.offsets = np.zeros(self.npatch + 1, dtype=np.int64)
        self.boxes = np.zeros((self.npatch, 4), dtype=np.int32)
        self.peers = np.zeros(self.npatch * (2 if dim == 1 else 4), dtype=np.int32)
        check(lib.nest_exchange_layout(self._h, self.offsets.ctypes.data_as(C.POINTER(C.c_longlong)),
                                       self.boxes.ctypes.data_as(C.POINTER(C.c_int)),
                                       self.peers.ctypes.data_as(C.POINTER(C.c_int))), "nest_exchange_layout")

    def close(self):
        if getattr(self, "_h", None):
            lib.nest_exchange_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def size(self) -> int:
        return int(self.offsets[-1])

    def patch_view(self, data: np.ndarray, p: int) -> np.ndarray:
        """[nvars, ext0(, ext1)] view of patch p inside the flat array."""
        s0, s1, n0, n1 = self.boxes[p]
        blk = data[self.offsets[p]:self.offsets[p + 1]]
        if self.dim == 1:
            return blk.reshape(self.nvars, n0 + 2 * self.halo)
        return blk.reshape(self.nvars, n0 + 2 * self.halo, n1 + 2 * self.halo)

    def execute_device(self, ptr: int, precision: int = A.F64, stream: int | None = None):
        check(lib.nest_exchange_execute(self._h, C.c_void_p(ptr), precision, C.c_void_p(stream) if stream else None),
              "nest_exchange_execute")
