"""Host logic of the x-slab decomposition (nest_b200/shard.py) on CPU.

The slabs here are the oracle's stage run on numpy arrays in the order the
device kernels follow (cut sides' ghost rows left to the exchange, speeds
max-reduced across slabs before stage 1), so a run on several slabs -- in
one process or as gloo ranks -- must equal the one-domain oracle run bit for
bit.  This covers the slab split, neighbour and tag bookkeeping, the message
order for two ranks (both neighbours the same rank) and the speed reduction.
"""
from __future__ import annotations

import contextlib
import os
import socket

import numpy as np
import pytest
import torch

from nest_b200.problems import kelvin_helmholtz, riemann_2d
from nest_b200.shard import SlabDomain, slab_range, slab_rows

G = 1.4


class OracleSlab:
    """CPU slab: the oracle's 2D stage on rows x0 .. x0+n of the domain."""

    def __init__(self, orc, U_slab, n, ny, dx, dy, bc, lo_ex, hi_ex):
        self.orc, self.n, self.ny, self.dx, self.dy, self.bc = orc, n, ny, dx, dy, bc
        self.lo_ex, self.hi_ex = lo_ex, hi_ex
        self.U = np.ascontiguousarray(U_slab, dtype=np.float64)
        self.U1 = np.zeros_like(self.U)
        self.tU, self.tU1 = torch.from_numpy(self.U), torch.from_numpy(self.U1)
        self.fill(self.U)
        self.words = torch.zeros(2, dtype=torch.int64)
        self._speeds()

    def fill(self, U):
        """Ghost fill of the slab's own sides (cut sides keep the exchanged rows)."""
        keep_lo = U[:, :2, :].copy() if self.lo_ex else None
        keep_hi = U[:, self.n + 2:, :].copy() if self.hi_ex else None
        self.orc.fill_ghosts2d(U, self.n, self.ny, 2, self.bc)
        if keep_lo is not None:
            U[:, :2, :] = keep_lo
        if keep_hi is not None:
            U[:, self.n + 2:, :] = keep_hi

    def _speeds(self):
        sx, sy = self.orc.max_speeds2d(self.U, self.n, self.ny, 2, G)
        self.words.copy_(torch.from_numpy(np.array([sx, sy]).view(np.int64)))

    def stream(self):
        return contextlib.nullcontext()

    def speed_words(self):
        return self.words

    def edges(self, buf):
        from nest_b200.shard import Edges
        t = self.tU if buf == 0 else self.tU1
        n = self.n
        return Edges(t[:, 2:4, :], t[:, n:n + 2, :], t[:, 0:2, :], t[:, n + 2:n + 4, :])

    def stage(self, which, cfl, t_final):
        n, ny = self.n, self.ny
        if which == 1:
            sx, sy = np.array(self.words.numpy()).view(np.float64)
            self.dt = self.orc.dt2d(float(sx), float(sy), self.dx, self.dy, cfl)
            self.fill(self.U)
            self.U1[...] = self.orc.stage2d(self.U, n, ny, 2, self.dt / self.dx, self.dt / self.dy, G)
            self.fill(self.U1)
        else:
            Us = self.orc.stage2d(self.U1, n, ny, 2, self.dt / self.dx, self.dt / self.dy, G)
            self.U[:, 2:-2, 2:-2] = 0.5 * (self.U[:, 2:-2, 2:-2] + Us[:, 2:-2, 2:-2])
            self.fill(self.U)
            self._speeds()


def make_slabs(orc, U, nx, ny, bc, parts, ids):
    periodic = bc == 0
    out = []
    for k in ids:
        x0, n = slab_range(nx, parts, k)
        lo_ex = parts > 1 and (periodic or k > 0)
        hi_ex = parts > 1 and (periodic or k < parts - 1)
        out.append(OracleSlab(orc, slab_rows(U, x0, n), n, ny, 1.0 / nx, 1.0 / ny, bc, lo_ex, hi_ex))
    return out


def one_domain(orc, U, nx, ny, bc, nsteps):
    U = U.copy()
    orc.run2d(U, nx, ny, 2, 1.0 / nx, 1.0 / ny, G, 0.4, nsteps=nsteps, bc=bc)
    return U[:, 2:-2, 2:-2]


def test_slab_range_matches_subspace():
    # subspace(): the first total % parts pieces carry one extra cell, contiguous cover
    for total, parts in [(10, 3), (7, 7), (4096, 8), (13, 2)]:
        spans = [slab_range(total, parts, k) for k in range(parts)]
        assert spans[0][0] == 0 and sum(n for _, n in spans) == total
        assert all(spans[k][0] + spans[k][1] == spans[k + 1][0] for k in range(parts - 1))
        assert [n for _, n in spans] == [total // parts + (1 if k < total % parts else 0) for k in range(parts)]


@pytest.mark.parametrize("bc,parts", [(0, 3), (1, 3), (0, 2), (1, 4)])
def test_local_slabs_equal_one_domain(oracle, bc, parts):
    nx, ny, nsteps = 23, 12, 6
    U = kelvin_helmholtz(nx, ny, seed=5) if bc == 0 else riemann_2d(nx, ny)
    slabs = make_slabs(oracle, U, nx, ny, bc, parts, range(parts))
    dom = SlabDomain(slabs, list(range(parts)), parts, periodic=(bc == 0))
    dom.step(nsteps, 0.4)
    got = np.concatenate([s.U[:, 2:-2, 2:-2] for s in slabs], axis=1)
    assert np.array_equal(got, one_domain(oracle, U, nx, ny, bc, nsteps))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, bc, nx, ny, nsteps, outdir):
    import datetime

    import torch.distributed as dist

    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc = Oracle()
        orc.set_threads(1)
        U = kelvin_helmholtz(nx, ny, seed=9) if bc == 0 else riemann_2d(nx, ny)
        (slab,) = make_slabs(orc, U, nx, ny, bc, world, [rank])
        dom = SlabDomain([slab], [rank], world, periodic=(bc == 0), group=dist.group.WORLD)
        dom.step(nsteps, 0.4)
        np.save(os.path.join(outdir, f"slab{rank}.npy"), slab.U[:, 2:-2, 2:-2])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("bc,world", [(0, 2), (1, 2), (0, 3)])
def test_gloo_ranks_equal_one_domain(oracle, tmp_path, bc, world):
    import torch.multiprocessing as mp
    nx, ny, nsteps = 17, 10, 5
    mp.start_processes(_rank_main, args=(world, _free_port(), bc, nx, ny, nsteps, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    got = np.concatenate([np.load(tmp_path / f"slab{r}.npy") for r in range(world)], axis=1)
    U = kelvin_helmholtz(nx, ny, seed=9) if bc == 0 else riemann_2d(nx, ny)
    assert np.array_equal(got, one_domain(oracle, U, nx, ny, bc, nsteps))


def test_native_driver_neighbours():
    """Neighbour ranks of the native slab driver: periodic rings (a one-slab
    domain is its own neighbour on both sides), open chains end in -1."""
    from nest_b200.shard import native_peers
    assert native_peers(0, 1, True) == (0, 0)
    assert native_peers(0, 1, False) == (-1, -1)
    assert [native_peers(k, 3, True) for k in range(3)] == [(2, 1), (0, 2), (1, 0)]
    assert [native_peers(k, 3, False) for k in range(3)] == [(-1, 1), (0, 2), (1, -1)]
    assert native_peers(0, 2, True) == (1, 1) and native_peers(1, 2, True) == (0, 0)
