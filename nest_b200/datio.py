"""nest's text snapshot formats and restartable checkpoints (C ABI in
include/nest_b200.h, implemented in nest_b200/csrc/datio.cpp).

write_dat_1d / write_dat_2d write a host state exactly as nest's examples do
(examples/sod1d/sod1d.cpp:50-91, examples/sod2d/sod2d.cpp:58-152) for a
given patch grid; ``dat_name`` builds nest's file names."""
from __future__ import annotations

import os

import numpy as np

from ._capi import check, lib


def dat_name(kind: str, step: int) -> str:
    """nest's snapshot file names: "sod" -> sod_0003.dat, "sod2d" ->
    sod2d_0003.dat, "sod2d_xslice" -> sod2d_xslice_0003.dat."""
    return f"{kind}_{step:04d}.dat"


def write_dat_1d(path, U, npatch: int = 1, x_min: float = 0.0, x_max: float = 1.0, gamma: float = 1.4,
                 time: float = 0.0, halo: int = 2):
    U = np.ascontiguousarray(U, dtype=np.float64)
    n = U.shape[1] - 2 * halo
    check(lib.nest_write_dat_1d(os.fsencode(path), U.ctypes.data, n, halo, npatch, x_min, x_max, gamma, time),
          "nest_write_dat_1d")


def write_dat_2d(path, U, npx: int = 1, npy: int = 1, x_min: float = 0.0, x_max: float = 1.0, y_min: float = 0.0,
                 y_max: float = 1.0, gamma: float = 1.4, time: float = 0.0, xslice: bool = False):
    U = np.ascontiguousarray(U, dtype=np.float64)
    nx, ny = U.shape[1] - 4, U.shape[2] - 4
    check(lib.nest_write_dat_2d(os.fsencode(path), U.ctypes.data, nx, ny, npx, npy, x_min, x_max, y_min, y_max,
                                gamma, time, int(xslice)), "nest_write_dat_2d")
