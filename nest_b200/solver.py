"""Host-side mirror of nest's solver interface over the C ABI.

``Euler1DGPU`` mirrors nest's euler1d_solver_t / euler1d_gpu_* ABI
(src/backend_cuda/euler1d_solver.hpp:16-87): same methods, same SoA-with-halo
host layout [var * n_total + i], same periodic boundary and run-from-zero
semantics of run()/run_timed().

``Solver`` is the general 1D/2D handle (FP64 plain form or FP32 form).
Host arrays are numpy; device tensors (torch) can be passed to
upload_device/download_device by pointer.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from ._capi import check, lib


class Euler1DGPU:
    """nest's 1D CUDA solver interface (periodic; FP64; bit-exact with its CPU path)."""

    def __init__(self, n_interior: int, n_halo: int, dx: float, gamma: float):
        self.n_interior, self.n_halo, self.dx, self.gamma = n_interior, n_halo, dx, gamma
        self.n_total = n_interior + 2 * n_halo
        self._h = lib.euler1d_gpu_create(n_interior, n_halo, dx, gamma)
        if not self._h:
            raise A.NestError(1, "euler1d_gpu_create", A.last_error())

    def _status(self, where):
        check(lib.euler1d_gpu_status(self._h), where)

    def close(self):
        if getattr(self, "_h", None):
            lib.euler1d_gpu_destroy(self._h)
            self._h = None

    __del__ = close

    def set_bc(self, bc: int):
        check(lib.euler1d_gpu_set_bc(self._h, bc), "euler1d_gpu_set_bc")

    def upload(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.size == 3 * self.n_total
        lib.euler1d_gpu_upload(self._h, U.ctypes.data_as(C.POINTER(C.c_double)))
        self._status("euler1d_gpu_upload")

    def download(self) -> np.ndarray:
        U = np.zeros((3, self.n_total))
        lib.euler1d_gpu_download(self._h, U.ctypes.data_as(C.POINTER(C.c_double)))
        self._status("euler1d_gpu_download")
        return U

    def compute_dt(self, cfl: float) -> float:
        dt = lib.euler1d_gpu_compute_dt(self._h, cfl)
        self._status("euler1d_gpu_compute_dt")
        return dt

    def rk2_step(self, dt: float):
        lib.euler1d_gpu_rk2_step(self._h, dt)
        self._status("euler1d_gpu_rk2_step")

    def run(self, t_final: float, cfl: float) -> int:
        n = lib.euler1d_gpu_run(self._h, t_final, cfl)
        self._status("euler1d_gpu_run")
        return n

    def run_timed(self, t_final: float, cfl: float):
        steps = C.c_int(0)
        ms = lib.euler1d_gpu_run_timed(self._h, t_final, cfl, C.byref(steps))
        self._status("euler1d_gpu_run_timed")
        return ms, steps.value


class Solver:
    """One domain on the device (see nest_solver_* in include/nest_b200.h)."""

    def __init__(self, dim: int, nx: int, ny: int = 1, dx: float = None, dy: float = None,
                 gamma: float = 1.4, bc=(A.BC_OUTFLOW, A.BC_OUTFLOW), precision: int = A.F64,
                 flags: int = 0, halo: int = 2, stream: int | None = None):
        if isinstance(bc, int):
            bc = (bc, bc)
        dx = dx if dx is not None else 1.0 / nx
        dy = dy if dy is not None else (1.0 / ny if dim == 2 else dx)
        self.dim, self.nx, self.ny, self.halo = dim, nx, ny, halo
        self.dx, self.dy, self.gamma, self.precision = dx, dy, gamma, precision
        self.dtype = np.float64 if precision == A.F64 else np.float32
        self.nvars = 3 if dim == 1 else 4
        d = A.SolverDesc(dim, nx, ny, halo, dx, dy, gamma, bc[0], bc[1], precision, flags,
                         C.c_void_p(stream) if stream else None)
        h = C.c_void_p()
        check(lib.nest_solver_create(C.byref(d), C.byref(h)), "nest_solver_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.nest_solver_destroy(self._h)
            self._h = None

    __del__ = close

    def shape(self, layout: int = A.LAYOUT_EXTENDED):
        g = 2 * self.halo if layout == A.LAYOUT_EXTENDED else 0
        if self.dim == 1:
            return (3, self.nx + g)
        return (4, self.nx + g, self.ny + g)

    def upload(self, U: np.ndarray, layout: int = A.LAYOUT_EXTENDED):
        U = np.ascontiguousarray(U, dtype=self.dtype)
        assert U.shape == self.shape(layout), (U.shape, self.shape(layout))
        check(lib.nest_solver_upload(self._h, U.ctypes.data, layout), "nest_solver_upload")

    def download(self, layout: int = A.LAYOUT_EXTENDED) -> np.ndarray:
        U = np.zeros(self.shape(layout), dtype=self.dtype)
        check(lib.nest_solver_download(self._h, U.ctypes.data, layout), "nest_solver_download")
        return U

    def upload_device(self, ptr: int, layout: int = A.LAYOUT_EXTENDED):
        check(lib.nest_solver_upload_device(self._h, C.c_void_p(ptr), layout), "nest_solver_upload_device")

    def download_device(self, ptr: int, layout: int = A.LAYOUT_EXTENDED):
        check(lib.nest_solver_download_device(self._h, C.c_void_p(ptr), layout), "nest_solver_download_device")

    def step(self, nsteps: int, cfl: float):
        check(lib.nest_solver_step(self._h, nsteps, cfl), "nest_solver_step")

    def step_profiled(self, nsteps: int, cfl: float):
        """nsteps steps with a CUDA event between kernels; returns
        (stage-1 ms per launch, stage-2 ms per launch, total span ms)."""
        ms = np.zeros(2 * nsteps, dtype=np.float32)
        tot = C.c_float(0)
        check(lib.nest_solver_step_profiled(self._h, nsteps, cfl, ms.ctypes.data_as(C.POINTER(C.c_float)),
                                            C.byref(tot)), "nest_solver_step_profiled")
        return ms[0::2].astype(np.float64), ms[1::2].astype(np.float64), float(tot.value)

    def step_dt(self, nsteps: int, dt: float):
        check(lib.nest_solver_step_dt(self._h, nsteps, dt), "nest_solver_step_dt")

    def run_to(self, t_final: float, cfl: float, max_steps: int = 0) -> int:
        n = C.c_int(0)
        check(lib.nest_solver_run_to(self._h, t_final, cfl, max_steps, C.byref(n)), "nest_solver_run_to")
        return n.value

    def compute_dt(self, cfl: float) -> float:
        dt = C.c_double(0)
        check(lib.nest_solver_compute_dt(self._h, cfl, C.byref(dt)), "nest_solver_compute_dt")
        return dt.value

    def time(self):
        t, s = C.c_double(0), C.c_int(0)
        check(lib.nest_solver_time(self._h, C.byref(t), C.byref(s)), "nest_solver_time")
        return t.value, s.value

    def reset_time(self):
        check(lib.nest_solver_reset_time(self._h), "nest_solver_reset_time")

    def totals(self) -> np.ndarray:
        out = np.zeros(4)
        check(lib.nest_solver_totals(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "nest_solver_totals")
        return out

    def repairs(self) -> int:
        n = C.c_uint(0)
        check(lib.nest_solver_repairs(self._h, C.byref(n)), "nest_solver_repairs")
        return n.value

    def sync(self):
        check(lib.nest_solver_sync(self._h), "nest_solver_sync")

    def set_tiling(self, rows_per_tile: int, warps_per_block: int):
        check(lib.nest_solver_set_tiling(self._h, rows_per_tile, warps_per_block), "nest_solver_set_tiling")

    def freeze_dts(self, dts: np.ndarray):
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        check(lib.nest_solver_set_dt_sequence(self._h, dts.ctypes.data_as(C.POINTER(C.c_double)), len(dts), 0),
              "nest_solver_set_dt_sequence")

    def record_dts(self, n: int):
        check(lib.nest_solver_set_dt_sequence(self._h, None, n, 1), "nest_solver_set_dt_sequence")

    def clear_dts(self):
        check(lib.nest_solver_set_dt_sequence(self._h, None, 0, 2), "nest_solver_set_dt_sequence")

    def recorded_dts(self, n: int) -> np.ndarray:
        out = np.zeros(n)
        check(lib.nest_solver_get_dts(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), n), "nest_solver_get_dts")
        return out

    def state_ptr(self):
        p, pitch, vs = C.c_void_p(), C.c_longlong(), C.c_longlong()
        check(lib.nest_solver_state_ptr(self._h, C.byref(p), C.byref(pitch), C.byref(vs)), "nest_solver_state_ptr")
        return p.value, pitch.value, vs.value

    # -- stage-level driving (sharded domains) --------------------------------
    def set_exchange_sides(self, xlo: bool, xhi: bool):
        """Mark x sides whose ghost rows a halo exchange fills (the kernels
        leave them alone)."""
        check(lib.nest_solver_set_exchange_sides(self._h, int(xlo), int(xhi)), "nest_solver_set_exchange_sides")

    def stage(self, which: int, cfl: float, t_final: float = 0.0):
        """Enqueue stage 1 (U -> U1, derives dt from the speed slot) or stage 2
        (U1 -> U, reduces the next step's wave speeds) of the current step."""
        check(lib.nest_solver_stage(self._h, which, cfl, t_final), "nest_solver_stage")

    def speed_slot_ptr(self) -> int:
        p = C.c_void_p()
        check(lib.nest_solver_speed_slot(self._h, C.byref(p)), "nest_solver_speed_slot")
        return p.value

    def stage_ptr(self) -> int:
        p = C.c_void_p()
        check(lib.nest_solver_stage_ptr(self._h, C.byref(p)), "nest_solver_stage_ptr")
        return p.value

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        check(lib.nest_solver_stream(self._h, C.byref(p)), "nest_solver_stream")
        return p.value or 0

    # -- on-disk formats ------------------------------------------------------
    def write_dat(self, path, npx: int = 1, npy: int = 1, x_min: float = 0.0, x_max: float = 1.0,
                  y_min: float = 0.0, y_max: float = 1.0, xslice: bool = False):
        """nest's text snapshot of the current state and time (patch grid npx x npy)."""
        import os
        check(lib.nest_solver_write_dat(self._h, os.fsencode(path), npx, npy, x_min, x_max, y_min, y_max,
                                        int(xslice)), "nest_solver_write_dat")

    def save(self, path):
        """Restartable checkpoint: state, time and step count."""
        import os
        check(lib.nest_solver_save(self._h, os.fsencode(path)), "nest_solver_save")

    def load(self, path):
        import os
        check(lib.nest_solver_load(self._h, os.fsencode(path)), "nest_solver_load")

    def set_time(self, time: float, steps: int = 0):
        check(lib.nest_solver_set_time(self._h, time, steps), "nest_solver_set_time")
