"""nest's text snapshot formats: the library's writers against nest's own
write_output / write_output_2d / write_xslice (compiled from its sources in
oracle/_ref) on the same states and patch grids, byte for byte.  Host code
only (no GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from nest_b200.datio import dat_name, write_dat_1d, write_dat_2d
from nest_b200.problems import kelvin_helmholtz, prim_to_cons_1d, sod_1d


def _state_1d(n, seed):
    rng = np.random.default_rng(seed)
    rho = 0.5 + rng.random(n)
    u = rng.standard_normal(n)
    p = 0.1 + rng.random(n)
    U = prim_to_cons_1d(rho, u, p)
    U[2, 2 + n // 3] = 0.5 * U[0, 2 + n // 3] * (U[1, 2 + n // 3] / U[0, 2 + n // 3]) ** 2 - 1e-3  # p < 0: clamped
    return U


@pytest.mark.parametrize("n,npatch,seed", [(400, 4, 0), (37, 5, 1), (10, 1, 2)])
def test_write_dat_1d_matches_nest(ref, tmp_path, n, npatch, seed):
    U = _state_1d(n, seed)
    t = 0.123456789012345
    theirs = ref.write_sod1d(tmp_path, U, n, 2, npatch, 0.0, 1.0, 1.4, t, 7)
    ours = tmp_path / "ours.dat"
    write_dat_1d(ours, U, npatch, 0.0, 1.0, 1.4, t)
    assert ours.read_bytes() == theirs.read_bytes()
    assert theirs.name == dat_name("sod", 7)


def test_write_dat_1d_sod_state(ref, tmp_path):
    U = sod_1d(400)
    theirs = ref.write_sod1d(tmp_path, U, 400, 2, 4, 0.0, 1.0, 1.4, 0.0, 0)
    ours = tmp_path / "ours.dat"
    write_dat_1d(ours, U, 4)
    assert ours.read_bytes() == theirs.read_bytes()


@pytest.mark.parametrize("nx,ny,npx,npy", [(20, 12, 2, 2), (13, 9, 3, 2), (8, 8, 1, 1), (30, 7, 4, 3)])
def test_write_dat_2d_matches_nest(ref, tmp_path, nx, ny, npx, npy):
    U = kelvin_helmholtz(nx, ny, seed=nx)
    t = 0.05
    full, xs = ref.write_sod2d(tmp_path, U, nx, ny, npx, npy, 0.0, 1.0, 0.0, 0.1, 1.4, t, 3)
    o_full, o_xs = tmp_path / "o_full.dat", tmp_path / "o_xs.dat"
    write_dat_2d(o_full, U, npx, npy, 0.0, 1.0, 0.0, 0.1, 1.4, t)
    write_dat_2d(o_xs, U, npx, npy, 0.0, 1.0, 0.0, 0.1, 1.4, t, xslice=True)
    assert o_full.read_bytes() == full.read_bytes()
    assert o_xs.read_bytes() == xs.read_bytes()


def test_write_dat_rejects_bad_sizes(tmp_path):
    from nest_b200 import NestError
    with pytest.raises(NestError):
        write_dat_1d(tmp_path / "x.dat", np.ones((3, 8)), npatch=9)
    with pytest.raises(NestError):
        write_dat_2d(tmp_path / "no_such_dir" / "x.dat", np.ones((4, 8, 8)))
