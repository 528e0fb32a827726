"""Discrete adjoint with checkpointing (nest_adjoint_* in include/nest_b200.h)
and its torch.autograd.Function.

``Adjoint`` records a forward sweep of a periodic solver (1D FP64 and FP32,
2D FP64 and FP32) and maps the adjoint of the final conserved state to the
adjoint of the initial one with the same frozen dt sequence.
``EulerRollout1D`` / ``EulerRollout2D`` wrap it as autograd functions:
U_T = rollout(U_0), so that gradients of any torch loss of U_T flow back to
U_0 (and, through torch, to whatever produced U_0, e.g. the primitive fields
or an initial perturbation)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from ._capi import check, lib
from .solver import Solver

_vp, _i, _d = C.c_void_p, C.c_int, C.c_double
UNIFORM, BINOMIAL = 0, 1

A.bind({
    "nest_adjoint_create": (_i, [_vp, _i, _i, _i, C.POINTER(_vp)]),
    "nest_adjoint_destroy": (_i, [_vp]),
    "nest_adjoint_forward": (_i, [_vp, _d, C.POINTER(C.c_double)]),
    "nest_adjoint_backward": (_i, [_vp, _vp, _vp, _i]),
    "nest_adjoint_get_dts": (_i, [_vp, C.POINTER(C.c_double)]),
    "nest_adjoint_stats": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                C.POINTER(C.c_longlong)]),
})


class Adjoint:
    def __init__(self, solver: Solver, nsteps: int, policy: int = UNIFORM, param: int = 64):
        self.solver, self.nsteps = solver, nsteps
        h = C.c_void_p()
        check(lib.nest_adjoint_create(solver._h, nsteps, policy, param, C.byref(h)), "nest_adjoint_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.nest_adjoint_destroy(self._h)
            self._h = None

    __del__ = close

    def forward(self, cfl: float = 0.4, dts=None):
        if dts is not None:
            dts = np.ascontiguousarray(dts, dtype=np.float64)
            assert len(dts) == self.nsteps
            p = dts.ctypes.data_as(C.POINTER(C.c_double))
        else:
            p = None
        check(lib.nest_adjoint_forward(self._h, cfl, p), "nest_adjoint_forward")

    def backward(self, lam_final: np.ndarray) -> np.ndarray:
        """Adjoint of the final state -> adjoint of the initial state, as host
        arrays in the solver's extended layout (1D [3][n+2h], 2D [4][nx+4][ny+4])."""
        s = self.solver
        lam_final = np.ascontiguousarray(lam_final, dtype=s.dtype)
        if s.dim == 1:
            out = np.zeros_like(lam_final)
            check(lib.nest_adjoint_backward(self._h, lam_final.ctypes.data, out.ctypes.data, 0), "nest_adjoint_backward")
            return out
        _, pitch, vs = s.state_ptr()
        rows = s.nx + 4
        dev = np.zeros(4 * vs, dtype=s.dtype)
        for k in range(4):
            dev[k * vs:k * vs + rows * pitch].reshape(rows, pitch)[:, :s.ny + 4] = lam_final[k]
        res = np.zeros_like(dev)
        check(lib.nest_adjoint_backward(self._h, dev.ctypes.data, res.ctypes.data, 0), "nest_adjoint_backward")
        out = np.zeros_like(lam_final)
        for k in range(4):
            out[k] = res[k * vs:k * vs + rows * pitch].reshape(rows, pitch)[:, :s.ny + 4]
        return out

    def backward_device(self, lam_final_ptr: int, lam_initial_ptr: int):
        check(lib.nest_adjoint_backward(self._h, C.c_void_p(lam_final_ptr), C.c_void_p(lam_initial_ptr), 1),
              "nest_adjoint_backward")

    def dts(self) -> np.ndarray:
        out = np.zeros(self.nsteps)
        check(lib.nest_adjoint_get_dts(self._h, out.ctypes.data_as(C.POINTER(C.c_double))), "nest_adjoint_get_dts")
        return out

    def stats(self) -> dict:
        f, b = C.c_double(), C.c_double()
        rc, sb = C.c_longlong(), C.c_longlong()
        check(lib.nest_adjoint_stats(self._h, C.byref(f), C.byref(b), C.byref(rc), C.byref(sb)), "nest_adjoint_stats")
        return {"forward_ms": f.value, "backward_ms": b.value, "recomputed_steps": rc.value,
                "checkpoint_bytes": sb.value}


def _autograd_function():
    import torch

    class EulerRollout1D(torch.autograd.Function):
        """U_T = rollout(U_0) for a periodic 1D FP64 solver.

        U0: float64 CUDA tensor [3, n] (interior conserved state rho, rho u, E).
        The forward pass records dts (CFL) or uses `dts`; the backward pass
        runs the checkpointed discrete adjoint with those dts."""

        @staticmethod
        def forward(ctx, U0, nsteps: int, cfl: float = 0.4, policy: int = UNIFORM, param: int = 64,
                     dts=None, gamma: float = 1.4):
            n = U0.shape[1]
            s = Solver(1, n, bc=A.BC_PERIODIC, gamma=gamma, flags=A.FLAG_NO_RESIDENT)
            U0c = U0.detach().contiguous()
            torch.cuda.current_stream().synchronize()
            s.upload_device(U0c.data_ptr(), A.LAYOUT_INTERIOR)
            adj = Adjoint(s, nsteps, policy, param)
            adj.forward(cfl, dts)
            UT = torch.empty_like(U0c)
            s.download_device(UT.data_ptr(), A.LAYOUT_INTERIOR)
            ctx.adj, ctx.solver, ctx.n = adj, s, n
            return UT

        @staticmethod
        def backward(ctx, gUT):
            n = ctx.n
            lam = torch.zeros((3, n + 4), dtype=torch.float64, device=gUT.device)
            lam[:, 2:-2] = gUT
            lam0 = torch.empty_like(lam)
            torch.cuda.current_stream().synchronize()
            ctx.adj.backward_device(lam.data_ptr(), lam0.data_ptr())
            return lam0[:, 2:-2].contiguous(), None, None, None, None, None, None

    return EulerRollout1D


def _autograd_function_2d():
    import torch

    class EulerRollout2D(torch.autograd.Function):
        """U_T = rollout(U_0) for a periodic 2D solver, FP64 (float64 tensor)
        or the FP32 form (float32 tensor).

        U0: CUDA tensor [4, nx, ny] (interior conserved state rho, rho u,
        rho v, E; y fastest).  The forward pass records dts (CFL) or uses
        `dts`; the backward pass runs the checkpointed discrete adjoint of the
        2D stage (uniform or binomial snapshots) with those dts."""

        @staticmethod
        def forward(ctx, U0, nsteps: int, cfl: float = 0.4, policy: int = BINOMIAL, param: int = 64,
                    dts=None, gamma: float = 1.4):
            _, nx, ny = U0.shape
            prec = A.F64 if U0.dtype == torch.float64 else A.F32
            s = Solver(2, nx, ny, bc=A.BC_PERIODIC, gamma=gamma, precision=prec)
            U0c = U0.detach().contiguous()
            torch.cuda.current_stream().synchronize()
            s.upload_device(U0c.data_ptr(), A.LAYOUT_INTERIOR)
            adj = Adjoint(s, nsteps, policy, param)
            adj.forward(cfl, dts)
            UT = torch.empty_like(U0c)
            s.download_device(UT.data_ptr(), A.LAYOUT_INTERIOR)
            ctx.adj, ctx.solver, ctx.shape = adj, s, (nx, ny)
            return UT

        @staticmethod
        def backward(ctx, gUT):
            nx, ny = ctx.shape
            _, pitch, vs = ctx.solver.state_ptr()
            # adjoint arrays in the solver's device layout: plane k at k * vs,
            # row i (-2 .. nx+1) at (i + 2) * pitch, column j at j + 2
            lam = torch.zeros(4 * vs, dtype=gUT.dtype, device=gUT.device)
            planes = lam.view(4, vs)[:, :(nx + 4) * pitch].view(4, nx + 4, pitch)
            planes[:, 2:nx + 2, 2:ny + 2] = gUT
            lam0 = torch.empty_like(lam)
            torch.cuda.current_stream().synchronize()
            ctx.adj.backward_device(lam.data_ptr(), lam0.data_ptr())
            g0 = lam0.view(4, vs)[:, :(nx + 4) * pitch].view(4, nx + 4, pitch)[:, 2:nx + 2, 2:ny + 2]
            return g0.contiguous(), None, None, None, None, None, None

    return EulerRollout2D


class _Lazy:
    fn = None
    fn2 = None


def rollout_1d(U0, nsteps: int, cfl: float = 0.4, policy: int = UNIFORM, param: int = 64, dts=None,
               gamma: float = 1.4):
    """Differentiable 1D periodic rollout (torch); see EulerRollout1D."""
    if _Lazy.fn is None:
        _Lazy.fn = _autograd_function()
    return _Lazy.fn.apply(U0, nsteps, cfl, policy, param, dts, gamma)


def rollout_2d(U0, nsteps: int, cfl: float = 0.4, policy: int = BINOMIAL, param: int = 64, dts=None,
               gamma: float = 1.4):
    """Differentiable 2D periodic rollout (torch); see EulerRollout2D."""
    if _Lazy.fn2 is None:
        _Lazy.fn2 = _autograd_function_2d()
    return _Lazy.fn2.apply(U0, nsteps, cfl, policy, param, dts, gamma)
