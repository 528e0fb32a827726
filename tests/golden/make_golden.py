"""Regenerate the golden fixtures from nest's own CPU code.

Runs in the build container only (it needs oracle/_ref/libnest_ref.so, built
by oracle/Makefile from the nest source tree).  Outputs, all small:
  sod100_periodic.npy   final state of run_cpu_sod (tests/test_euler_cuda.cpp:49-185):
                        periodic Sod, N=100, t=0.1, CFL 0.3, SoA 3 x 104
  sod1d_final.npy       last output of the sod1d example (examples/sod1d/sod1d.cpp):
                        columns x rho u p e at t=0.2, N=400, 4 periodic patches
  sod2d_final.npz       last output of the sod2d example (examples/sod2d/sod2d.cpp):
                        columns x y rho u v p at t=0.2, 200 x 20 cells, 2 x 2 periodic patches
  known_answers.json    nest's numerics on the inputs of tests/test_euler.cpp:54-237
                        and on a seeded set of random states

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import glob
import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
from oracle.oracle import Reference  # noqa: E402


def main():
    ref = Reference()
    np.save(HERE / "sod100_periodic.npy", ref.run_cpu_sod(100, 0.1, 0.3))

    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            rc = ref.L.ref_sod1d_main()
        finally:
            os.chdir(cwd)
        assert rc == 0, rc
        last = sorted(glob.glob(os.path.join(td, "sod_*.dat")))[-1]
        np.save(HERE / "sod1d_final.npy", np.loadtxt(last, comments="#"))

    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            rc = ref.L.ref_sod2d_main()
        finally:
            os.chdir(cwd)
        assert rc == 0, rc
        outs = sorted(f for f in glob.glob(os.path.join(td, "sod2d_*.dat")) if "xslice" not in f)
        a = np.loadtxt(outs[-1], comments="#").astype(np.float64)
        np.savez_compressed(HERE / "sod2d_final.npz", x=a[:, 0], y=a[:, 1], rho=a[:, 2], u=a[:, 3], v=a[:, 4],
                            p=a[:, 5])

    import ctypes as C
    dp = C.POINTER(C.c_double)

    def arr(v):
        return np.ascontiguousarray(v, dtype=np.float64)

    rng = np.random.default_rng(7)
    cases = []
    for _ in range(64):
        WL = arr([rng.uniform(0.05, 2.0), rng.normal(0, 2.0), rng.uniform(0.01, 3.0)])
        WR = arr([rng.uniform(0.05, 2.0), rng.normal(0, 2.0), rng.uniform(0.01, 3.0)])
        cases.append({"WL": WL.tolist(), "WR": WR.tolist(), "F": ref.hlle_flux(1.4, WL, WR).tolist()})
    ka = {
        "eos_pressure_1_0_2.5": ref.L.ref_pressure(1.4, 1.0, 0.0, 2.5),
        "eos_total_energy_1_1_1": ref.L.ref_total_energy(1.4, 1.0, 1.0, 1.0),
        "eos_sound_speed_1_1": ref.L.ref_sound_speed(1.4, 1.0, 1.0),
        "hlle_stationary": ref.hlle_flux(1.4, arr([1, 0, 1]), arr([1, 0, 1])).tolist(),
        "hlle_supersonic": ref.hlle_flux(1.4, arr([1, 10, 1]), arr([1, 10, 1])).tolist(),
        "hlle_random": cases,
    }
    (HERE / "known_answers.json").write_text(json.dumps(ka, indent=1))
    print("wrote", sorted(p.name for p in HERE.iterdir()))


if __name__ == "__main__":
    main()
