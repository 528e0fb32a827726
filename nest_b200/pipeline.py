"""Device pipeline executor over nest's per-patch storage (nest_pipeline_* in
include/nest_b200.h): the device counterpart of nest's pipeline_t /
execute (include/nest/pipeline.hpp) and of the stage loops of its sod1d
example (examples/sod1d/sod1d.cpp:219-302)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from ._capi import check, lib
from .exchange import PeriodicExchange

_vp, _i, _d = C.c_void_p, C.c_int, C.c_double
A.bind({
    "nest_pipeline_create": (_i, [_i, _i, _i, _i, _i, _i, _d, _d, _i, _i, C.POINTER(_vp)]),
    "nest_pipeline_destroy": (_i, [_vp]),
    "nest_pipeline_plan": (_i, [_vp, C.POINTER(_vp)]),
    "nest_pipeline_add": (_i, [_vp, _i, _i, _i, _i, _d]),
    "nest_pipeline_execute": (_i, [_vp, _vp, _vp]),
    "nest_pipeline_run": (_i, [_vp, _vp, _d, _i, C.POINTER(_i), _vp]),
    "nest_pipeline_clock": (_i, [_vp, C.POINTER(_d), C.POINTER(_d), C.POINTER(_i)]),
    "nest_pipeline_set_clock": (_i, [_vp, _d, _d, _i]),
    "nest_pipeline_buffer": (_i, [_vp, _i, C.POINTER(_vp)]),
})

EXCHANGE, EULER_RHS, COPY, AVERAGE, CFL_DT, CHECK, CLOCK = 1, 2, 3, 4, 5, 6, 7
STATE = 0  # buffer 0: the caller's state


class Pipeline:
    """Stages over every patch of a periodic patch grid; buffer 0 is the
    caller's device state, 1..nwork the pipeline's work arrays."""

    def __init__(self, dim: int, nx: int, npx: int, halo: int = 2, dx: float | None = None, gamma: float = 1.4,
                 limiter: int = 0, nwork: int = 3, ny: int = 1, npy: int = 1):
        h = C.c_void_p()
        dx = dx if dx is not None else 1.0 / nx
        check(lib.nest_pipeline_create(dim, nx, ny, npx, npy, halo, dx, gamma, limiter, nwork, C.byref(h)),
              "nest_pipeline_create")
        self._h = h
        self.dim, self.nx, self.halo = dim, nx, halo
        plan = C.c_void_p()
        check(lib.nest_pipeline_plan(h, C.byref(plan)), "nest_pipeline_plan")
        # layout of the storage (the plan is owned by the pipeline)
        self.layout = PeriodicExchange.__new__(PeriodicExchange)
        self.layout.dim, self.layout.nvars, self.layout.halo = dim, 3 if dim == 1 else 4, halo
        self.layout.npatch = npx * (npy if dim == 2 else 1)
        self.layout._h = None
        self.layout.offsets = np.zeros(self.layout.npatch + 1, dtype=np.int64)
        self.layout.boxes = np.zeros((self.layout.npatch, 4), dtype=np.int32)
        check(lib.nest_exchange_layout(plan, self.layout.offsets.ctypes.data_as(C.POINTER(C.c_longlong)),
                                       self.layout.boxes.ctypes.data_as(C.POINTER(C.c_int)), None),
              "nest_exchange_layout")

    def close(self):
        if getattr(self, "_h", None):
            lib.nest_pipeline_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def size(self) -> int:
        return int(self.layout.offsets[-1])

    def add(self, kind: int, src: int = STATE, dst: int = STATE, aux: int = STATE, param: float = 0.0):
        check(lib.nest_pipeline_add(self._h, kind, src, dst, aux, param), "nest_pipeline_add")
        return self

    def execute(self, ptr: int, stream: int | None = None):
        """All stages once on `stream` (default: the pipeline's own
        non-blocking stream).  Returns when they are enqueued: read the state
        after clock() (which waits) or a synchronize of that stream."""
        check(lib.nest_pipeline_execute(self._h, C.c_void_p(ptr), C.c_void_p(stream) if stream else None),
              "nest_pipeline_execute")

    def run(self, ptr: int, t_final: float, max_steps: int = 0, stream: int | None = None) -> int:
        n = C.c_int(0)
        check(lib.nest_pipeline_run(self._h, C.c_void_p(ptr), t_final, max_steps, C.byref(n),
                                    C.c_void_p(stream) if stream else None), "nest_pipeline_run")
        return n.value

    def clock(self):
        t, dt, s = C.c_double(), C.c_double(), C.c_int()
        check(lib.nest_pipeline_clock(self._h, C.byref(t), C.byref(dt), C.byref(s)), "nest_pipeline_clock")
        return t.value, dt.value, s.value

    def set_clock(self, time: float = 0.0, dt: float = 0.0, step: int = 0):
        check(lib.nest_pipeline_set_clock(self._h, time, dt, step), "nest_pipeline_set_clock")

    # -- host layout helpers (1D) ---------------------------------------------
    def scatter(self, U: np.ndarray) -> np.ndarray:
        """Global interior state [nvars][n] -> per-patch storage (halos zero)."""
        out = np.zeros(self.size)
        for p in range(self.layout.npatch):
            s0, _, n0, _ = self.layout.boxes[p]
            self.layout.patch_view(out, p)[:, self.halo:self.halo + n0] = U[:, s0:s0 + n0]
        return out

    def gather(self, data: np.ndarray) -> np.ndarray:
        """Per-patch storage -> global interior state [nvars][n]."""
        U = np.zeros((self.layout.nvars, self.nx))
        for p in range(self.layout.npatch):
            s0, _, n0, _ = self.layout.boxes[p]
            U[:, s0:s0 + n0] = self.layout.patch_view(data, p)[:, self.halo:self.halo + n0]
        return U


def sod1d_pipeline(nx: int, npx: int, cfl: float = 0.4, halo: int = 2, gamma: float = 1.4, limiter: int = 0,
                   check_every: int = 10) -> Pipeline:
    """nest's sod1d time step (examples/sod1d/sod1d.cpp:219-302) as stages:
    dt from the CFL rule, halos, U0 = U, U1 = U + dt L(U) with nest's patch
    right-hand side, U = U1, halos, U2 = U + dt L(U), U = 0.5 U0 + 0.5 U2,
    positivity check every `check_every` steps, clock."""
    p = Pipeline(1, nx, npx, halo=halo, gamma=gamma, limiter=limiter, nwork=3)
    p.add(CFL_DT, src=STATE, param=cfl)
    p.add(EXCHANGE, src=STATE)
    p.add(COPY, src=STATE, dst=1)
    p.add(EULER_RHS, src=STATE, dst=2)
    p.add(COPY, src=2, dst=STATE)
    p.add(EXCHANGE, src=STATE)
    p.add(EULER_RHS, src=STATE, dst=3)
    p.add(AVERAGE, src=1, aux=3, dst=STATE)
    if check_every > 0:
        p.add(CHECK, src=STATE, param=check_every)
    p.add(CLOCK)
    return p
