"""ctypes bindings for the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and the CPU-baseline leg of bench.py import this
module.  The product (nest_b200/) never does.

``Oracle``    wraps oracle/liboracle.so, the plain-C restatement of nest's CPU
              algorithm (oracle/euler_oracle.c).
``Reference`` wraps oracle/_ref/libnest_ref.so, nest's own CPU code compiled
              from its source tree by oracle/Makefile.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BC_PERIODIC, BC_OUTFLOW = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


# Where the nest source tree is looked for when NEST_REF is not set.
DEFAULT_REF = "/root/reference"


def build(quiet: bool = True) -> None:
    """Run oracle/Makefile (the system gcc-13 with OpenMP); nest's own sources
    are compiled into _ref/ when their tree is present (environment variable
    NEST_REF, else DEFAULT_REF)."""
    import subprocess

    ref = os.environ.get("NEST_REF", DEFAULT_REF)
    cmd = ["make", "-C", str(HERE)]
    if Path(ref, "examples", "sod1d", "euler1d.hpp").exists():
        cmd.append(f"REF={ref}")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


class Oracle:
    def __init__(self, path: str | os.PathLike | None = None):
        path = Path(path) if path else HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        self.L = L
        d, i = C.c_double, C.c_int
        sig = {
            "orc_set_threads": (None, [i]),
            "orc_set_limiter": (None, [i]),
            "orc_max_threads": (i, []),
            "orc_pressure": (d, [d, d, d, d]),
            "orc_total_energy": (d, [d, d, d, d]),
            "orc_sound_speed": (d, [d, d, d]),
            "orc_cons_to_prim": (None, [d, _dp, _dp]),
            "orc_prim_to_cons": (None, [d, _dp, _dp]),
            "orc_minmod": (d, [d, d]),
            "orc_mc": (d, [d, d]),
            "orc_limit": (d, [d, d, i]),
            "orc_plm": (None, [_dp, _dp, _dp, i, i, _dp, _dp]),
            "orc_hlle1d": (None, [d, _dp, _dp, _dp]),
            "orc1d_fill_ghosts": (None, [_dp, i, i, i]),
            "orc1d_stage": (None, [_dp, _dp, _dp, i, i, d, d, d]),
            "orc1d_max_speed": (d, [_dp, i, i, d]),
            "orc1d_rk2_step": (None, [_dp, _dp, _dp, _dp, i, i, d, d, d, i]),
            "orc1d_run": (i, [_dp, i, i, d, d, d, d, i, i, _dp, _dp, _dp]),
            "orc1d_patch_stage": (None, [_dp, _dp, _dp, i, i, d, d, d]),
            "orc_cons_to_prim2d": (None, [d, _dp, _dp]),
            "orc_prim_to_cons2d": (None, [d, _dp, _dp]),
            "orc_hlle2d": (None, [d, _dp, _dp, _dp]),
            "orc2d_fill_ghosts": (None, [_dp, i, i, i, i, i]),
            "orc2d_stage": (None, [_dp, _dp, _dp, i, i, i, d, d, d]),
            "orc2d_max_speeds": (None, [_dp, i, i, i, d, _dp, _dp]),
            "orc2d_dt_from_speeds": (d, [d, d, d, d, d]),
            "orc2d_rk2_step": (None, [_dp, _dp, _dp, _dp, i, i, i, d, d, d, d, i, i]),
            "orc2d_run": (i, [_dp, i, i, i, d, d, d, d, d, i, i, i, _dp, _dp, _dp]),
            "orc2d_totals": (None, [_dp, i, i, i, d, d, _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args

    def set_limiter(self, lim: int) -> None:
        """Limiter of the stage functions: 0 minmod (default), 1 MC, 2 none."""
        self.L.orc_set_limiter(int(lim))

    def set_threads(self, n: int) -> None:
        self.L.orc_set_threads(int(n))

    def max_threads(self) -> int:
        return int(self.L.orc_max_threads())

    # -- scalar numerics -------------------------------------------------
    def hlle1d(self, gamma, WL, WR):
        F = np.zeros(3)
        self.L.orc_hlle1d(gamma, _ptr(np.ascontiguousarray(WL, np.float64)),
                          _ptr(np.ascontiguousarray(WR, np.float64)), _ptr(F))
        return F

    def hlle2d(self, gamma, WL, WR):
        F = np.zeros(4)
        self.L.orc_hlle2d(gamma, _ptr(np.ascontiguousarray(WL, np.float64)),
                          _ptr(np.ascontiguousarray(WR, np.float64)), _ptr(F))
        return F

    # -- 1D ----------------------------------------------------------------
    def run1d(self, U, n, h, dx, gamma, cfl, t_final=0.0, nsteps=0, bc=BC_PERIODIC,
              dts_in=None, record_dts=False):
        """Advance U (SoA 3 x (n+2h), float64, in place).  Returns (steps, t, dts)."""
        assert U.shape == (3, n + 2 * h)
        cap = nsteps if nsteps > 0 else 1_000_000
        dts = np.zeros(cap) if record_dts else None
        t = C.c_double(0.0)
        steps = self.L.orc1d_run(_ptr(U), n, h, dx, gamma, cfl, t_final, nsteps, bc,
                                 _ptr(dts_in), _ptr(dts), C.byref(t))
        return steps, t.value, (dts[:steps] if record_dts else None)

    def stage1d(self, Uin, n, h, dx, dt, gamma):
        Uout = Uin.copy()
        W = np.zeros_like(Uin)
        self.L.orc1d_stage(_ptr(Uin), _ptr(Uout), _ptr(W), n, h, dx, dt, gamma)
        return Uout

    def max_speed1d(self, U, n, h, gamma):
        return float(self.L.orc1d_max_speed(_ptr(U), n, h, gamma))

    def patch_stage1d(self, Uin, n, h, dx, dt, gamma):
        Uout = np.zeros_like(Uin)
        W = np.zeros_like(Uin)
        self.L.orc1d_patch_stage(_ptr(Uin), _ptr(Uout), _ptr(W), n, h, dx, dt, gamma)
        return Uout

    def fill_ghosts1d(self, U, n, h, bc):
        self.L.orc1d_fill_ghosts(_ptr(U), n, h, bc)

    # -- 2D ----------------------------------------------------------------
    def run2d(self, U, nx, ny, h, dx, dy, gamma, cfl, t_final=0.0, nsteps=0,
              bc=BC_OUTFLOW, dts_in=None, record_dts=False):
        """Advance U (4 x (nx+2h) x (ny+2h), float64, in place).  bc is one
        condition for both axes or a (bc_x, bc_y) pair."""
        assert U.shape == (4, nx + 2 * h, ny + 2 * h)
        bcx, bcy = (bc, bc) if isinstance(bc, int) else bc
        cap = nsteps if nsteps > 0 else 1_000_000
        dts = np.zeros(cap) if record_dts else None
        t = C.c_double(0.0)
        steps = self.L.orc2d_run(_ptr(U), nx, ny, h, dx, dy, gamma, cfl, t_final,
                                 nsteps, bcx, bcy, _ptr(dts_in), _ptr(dts), C.byref(t))
        return steps, t.value, (dts[:steps] if record_dts else None)

    def fill_ghosts2d(self, U, nx, ny, h, bc):
        bcx, bcy = (bc, bc) if isinstance(bc, int) else bc
        self.L.orc2d_fill_ghosts(_ptr(U), nx, ny, h, bcx, bcy)

    def stage2d(self, Uin, nx, ny, h, dtdx, dtdy, gamma):
        Uout = Uin.copy()
        W = np.zeros_like(Uin)
        self.L.orc2d_stage(_ptr(Uin), _ptr(Uout), _ptr(W), nx, ny, h, dtdx, dtdy, gamma)
        return Uout

    def max_speeds2d(self, U, nx, ny, h, gamma):
        sx, sy = C.c_double(), C.c_double()
        self.L.orc2d_max_speeds(_ptr(U), nx, ny, h, gamma, C.byref(sx), C.byref(sy))
        return sx.value, sy.value

    def dt2d(self, sx, sy, dx, dy, cfl):
        return float(self.L.orc2d_dt_from_speeds(sx, sy, dx, dy, cfl))

    def totals2d(self, U, nx, ny, h, dx, dy):
        out = np.zeros(4)
        self.L.orc2d_totals(_ptr(U), nx, ny, h, dx, dy, _ptr(out))
        return out


class Reference:
    """nest's own CPU functions, compiled from its source tree into _ref/."""

    def __init__(self, path: str | os.PathLike | None = None):
        path = Path(path) if path else HERE / "_ref" / "libnest_ref.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (needs the nest source tree)")
        L = C.CDLL(str(path))
        self.L = L
        d, i = C.c_double, C.c_int
        sig = {
            "ref_pressure": (d, [d, d, d, d]),
            "ref_total_energy": (d, [d, d, d, d]),
            "ref_sound_speed": (d, [d, d, d]),
            "ref_cons_to_prim": (None, [d, _dp, _dp]),
            "ref_prim_to_cons": (None, [d, _dp, _dp]),
            "ref_minmod": (d, [d, d]),
            "ref_mc": (d, [d, d]),
            "ref_plm": (None, [_dp, _dp, _dp, i, _dp, _dp]),
            "ref_hlle_flux": (None, [d, _dp, _dp, _dp]),
            "ref_patch_stage": (None, [_dp, _dp, i, i, d, d, d]),
            "ref_exchange_1d": (i, [_dp, i, i, i, i]),
            "ref_exchange_2d": (i, [_dp, i, i, i, i, i, i]),
            "ref_patch_boxes_2d": (i, [i, i, i, i, _ip]),
            "ref_x_sweep": (None, [_dp, _dp, i, i, i, d, d, d, i]),
            "ref_y_sweep": (None, [_dp, _dp, i, i, i, d, d, d, i]),
            "ref_compute_dt_2d": (d, [_dp, i, i, i, d, d, d, d]),
            "ref_benchmark_cpu": (d, [i, d, _ip, _dp]),
            "ref_sod1d_main": (i, []),
            "ref_sod2d_main": (i, []),
            "ref_run_cpu_sod": (None, [i, d, d, _dp]),
            "ref_write_sod1d": (None, [_dp, i, i, i, d, d, d, d, i]),
            "ref_write_sod2d": (None, [_dp, i, i, i, i, d, d, d, d, d, d, i]),
            "ref_pipeline_euler1d": (None, [_dp, i, i, i, d, d, i, i, _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args

    def write_sod1d(self, directory, U, n, halo, npatch, x_min, x_max, gamma, time, step):
        """nest's write_output on state U; returns the path of the file it wrote."""
        U = np.ascontiguousarray(U, np.float64)
        cwd = os.getcwd()
        os.chdir(directory)
        try:
            self.L.ref_write_sod1d(_ptr(U), n, halo, npatch, x_min, x_max, gamma, time, step)
        finally:
            os.chdir(cwd)
        return Path(directory) / f"sod_{step:04d}.dat"

    def write_sod2d(self, directory, U, nx, ny, npx, npy, x_min, x_max, y_min, y_max, gamma, time, step):
        """nest's write_output_2d and write_xslice; returns both paths."""
        U = np.ascontiguousarray(U, np.float64)
        cwd = os.getcwd()
        os.chdir(directory)
        try:
            self.L.ref_write_sod2d(_ptr(U), nx, ny, npx, npy, x_min, x_max, y_min, y_max, gamma, time, step)
        finally:
            os.chdir(cwd)
        return Path(directory) / f"sod2d_{step:04d}.dat", Path(directory) / f"sod2d_xslice_{step:04d}.dat"

    def hlle_flux(self, gamma, WL, WR):
        F = np.zeros(3)
        self.L.ref_hlle_flux(gamma, _ptr(np.ascontiguousarray(WL, np.float64)),
                             _ptr(np.ascontiguousarray(WR, np.float64)), _ptr(F))
        return F

    def run_cpu_sod(self, n, t_final, cfl):
        U = np.zeros(3 * (n + 4))
        self.L.ref_run_cpu_sod(n, t_final, cfl, _ptr(U))
        return U.reshape(3, n + 4)

    def patch_stage(self, Uin, n, h, dx, dt, gamma):
        Uout = np.zeros_like(Uin)
        self.L.ref_patch_stage(_ptr(np.ascontiguousarray(Uin)), _ptr(Uout), n, h, dx, dt, gamma)
        return Uout

    def pipeline_euler1d(self, U, npatch, halo, gamma, cfl, nexec, limiter=0):
        """nest::execute of (dt reduce, exchange, euler_rhs compute) on nest's
        patches, nexec times, from the global interior state U [3][n];
        returns (final U, dts)."""
        U = np.ascontiguousarray(U, np.float64).copy()
        dts = np.zeros(nexec)
        self.L.ref_pipeline_euler1d(_ptr(U), U.shape[1], npatch, halo, gamma, cfl, limiter, nexec, _ptr(dts))
        return U, dts

    def benchmark_cpu(self, n_zones, t_final):
        steps = C.c_int(0)
        cps = C.c_double(0.0)
        ms = self.L.ref_benchmark_cpu(n_zones, t_final, C.byref(steps), C.byref(cps))
        return ms, steps.value, cps.value


def sod_ic_1d(n: int, h: int = 2, gamma: float = 1.4, x_disc: float = 0.5):
    """Sod state on cell centres x = (i - h + 0.5) dx, halos included
    (initialize_sod, examples/benchmark/benchmark_euler1d.cpp:53-77)."""
    dx = 1.0 / n
    nt = n + 2 * h
    U = np.zeros((3, nt))
    for i in range(nt):
        x = 0.0 + (i - h + 0.5) * dx
        if x < x_disc:
            rho, u, p = 1.0, 0.0, 1.0
        else:
            rho, u, p = 0.125, 0.0, 0.1
        ke = 0.5 * rho * u * u
        E = p / (gamma - 1.0) + ke
        U[0, i], U[1, i], U[2, i] = rho, rho * u, E
    return U
