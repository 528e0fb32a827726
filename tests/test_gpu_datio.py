"""Checkpoint / restart and snapshot writing through the solver."""
from __future__ import annotations

import numpy as np
import pytest

from nest_b200.problems import kelvin_helmholtz, riemann_2d, sod_1d

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,prec", [(1, "F64"), (2, "F64"), (2, "F32")])
def test_restart_continues_bit_for_bit(gpu, tmp_path, dim, prec):
    prec = getattr(gpu, prec)
    if dim == 1:
        mk = lambda: gpu.Solver(1, 300, bc=gpu.BC_OUTFLOW, flags=gpu.FLAG_NO_RESIDENT)
        U0 = sod_1d(300)
    else:
        mk = lambda: gpu.Solver(2, 96, 80, bc=gpu.BC_PERIODIC, precision=prec)
        U0 = kelvin_helmholtz(96, 80, seed=4).astype(np.float64 if prec == gpu.F64 else np.float32)
    a = mk()
    a.upload(U0)
    a.step(17, 0.4)
    a.save(tmp_path / "ck.bin")
    a.step(23, 0.4)
    b = mk()
    b.load(tmp_path / "ck.bin")
    assert b.time()[1] == 17
    b.step(23, 0.4)
    # interior (2D corner ghost cells are never read by the scheme and are not kept up to date)
    ia, ib = a.download(), b.download()
    if dim == 1:
        assert np.array_equal(ia, ib)
    else:
        assert np.array_equal(ia[:, 2:-2, 2:-2], ib[:, 2:-2, 2:-2])
    assert a.time() == b.time()


def test_load_rejects_mismatch(gpu, tmp_path):
    a = gpu.Solver(2, 32, 32)
    a.upload(riemann_2d(32, 32))
    a.save(tmp_path / "ck.bin")
    with pytest.raises(gpu.NestError):
        gpu.Solver(2, 32, 33).load(tmp_path / "ck.bin")
    with pytest.raises(gpu.NestError):
        gpu.Solver(2, 32, 32, precision=gpu.F32).load(tmp_path / "ck.bin")
    raw = bytearray((tmp_path / "ck.bin").read_bytes())
    raw[200] ^= 1
    (tmp_path / "bad.bin").write_bytes(bytes(raw))
    with pytest.raises(gpu.NestError):
        gpu.Solver(2, 32, 32).load(tmp_path / "bad.bin")


def test_solver_snapshot_equals_host_writer(gpu, tmp_path):
    from nest_b200.datio import write_dat_2d
    s = gpu.Solver(2, 40, 24, bc=gpu.BC_OUTFLOW)
    s.upload(riemann_2d(40, 24))
    s.step(5, 0.4)
    s.write_dat(tmp_path / "dev.dat", 2, 2, 0.0, 1.0, 0.0, 1.0)
    t, _ = s.time()
    write_dat_2d(tmp_path / "host.dat", s.download(), 2, 2, 0.0, 1.0, 0.0, 1.0, 1.4, t)
    assert (tmp_path / "dev.dat").read_bytes() == (tmp_path / "host.dat").read_bytes()
