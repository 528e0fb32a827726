"""x-slab decomposition on the device: several slabs of one domain on one GPU
(stage kernels with cut sides, halo rows moved by copies, speeds max-reduced)
equal the one-domain solver bit for bit, FP64 and FP32."""
from __future__ import annotations

import numpy as np
import pytest

from nest_b200.problems import kelvin_helmholtz, riemann_2d

pytestmark = pytest.mark.gpu


def run_slabs(gpu, U, nx, ny, bc, prec, parts, nsteps, t_final=0.0, flags=0):
    import torch
    from nest_b200.shard import gpu_domain, slab_rows
    dom, ranges = gpu_domain(nx, ny, bc=bc, precision=prec, flags=flags, local_slabs=parts)
    dt = np.float64 if prec == gpu.F64 else np.float32
    for s, (x0, n) in zip(dom.slabs, ranges):
        s.solver.upload(slab_rows(U, x0, n).astype(dt))
    dom.step(nsteps, 0.4, t_final)
    torch.cuda.synchronize()
    parts_out = [s.solver.download()[:, 2:-2, 2:-2] for s in dom.slabs]
    times = [s.solver.time() for s in dom.slabs]
    return np.concatenate(parts_out, axis=1), times


def run_one(gpu, U, nx, ny, bc, prec, nsteps, t_final=0.0, flags=0):
    s = gpu.Solver(2, nx, ny, bc=bc, precision=prec, flags=flags)
    s.upload(U.astype(np.float64 if prec == gpu.F64 else np.float32))
    if t_final > 0.0:
        s.run_to(t_final, 0.4, max_steps=nsteps)
    else:
        s.step(nsteps, 0.4)
    return s.download()[:, 2:-2, 2:-2], s.time()


@pytest.mark.parametrize("prec", ["F64", "F32"])
@pytest.mark.parametrize("bc,parts,nx,ny", [(0, 2, 130, 96), (1, 3, 201, 77), (0, 5, 97, 200), (1, 2, 64, 64)])
def test_slabs_equal_one_domain(gpu, prec, bc, parts, nx, ny):
    prec = getattr(gpu, prec)
    U = kelvin_helmholtz(nx, ny, seed=2) if bc == gpu.BC_PERIODIC else riemann_2d(nx, ny)
    got, times = run_slabs(gpu, U, nx, ny, bc, prec, parts, 25)
    want, t1 = run_one(gpu, U, nx, ny, bc, prec, 25)
    assert np.array_equal(got, want)
    assert all(t == t1 for t in times)


def test_slabs_stop_at_t_final(gpu):
    nx, ny = 96, 80
    U = riemann_2d(nx, ny)
    t_final = 0.01
    got, times = run_slabs(gpu, U, nx, ny, gpu.BC_OUTFLOW, gpu.F64, 3, 200, t_final=t_final)
    want, (t1, n1) = run_one(gpu, U, nx, ny, gpu.BC_OUTFLOW, gpu.F64, 200, t_final=t_final)
    assert np.array_equal(got, want)
    assert abs(t1 - t_final) <= 1e-15 and all(t == (t1, n1) for t in times)


def test_exchange_sides_checks(gpu):
    s1 = gpu.Solver(1, 64, bc=gpu.BC_PERIODIC)
    with pytest.raises(gpu.NestError):
        s1.set_exchange_sides(True, True)
    s2 = gpu.Solver(2, 32, 32, flags=gpu.FLAG_SPLIT_COMPAT)
    with pytest.raises(gpu.NestError):
        s2.set_exchange_sides(True, False)


@pytest.mark.parametrize("prec", ["F64", "F32"])
@pytest.mark.parametrize("bc,nx,ny,nsteps", [(0, 130, 96, 37), (1, 96, 80, 20)])
def test_native_driver_one_rank_equals_one_domain(gpu, prec, bc, nx, ny, nsteps):
    """The C++ slab driver (nest_slab_step: NCCL speed all-reduce and
    ghost-row send / recv on the solver's stream, 16-step CUDA graphs) on a
    one-rank domain: periodic x exchanges the slab's rows with itself through
    NCCL, outflow has no cut side.  The result equals the one-domain solver
    bit for bit (37 steps: two graph replays and five single steps)."""
    import torch
    from nest_b200.shard import gpu_domain, slab_rows
    prec = getattr(gpu, prec)
    U = kelvin_helmholtz(nx, ny, seed=5) if bc == gpu.BC_PERIODIC else riemann_2d(nx, ny)
    dom, ranges = gpu_domain(nx, ny, bc=bc, precision=prec, native=True)
    (slab,), ((x0, n),) = dom.slabs, ranges
    slab.solver.upload(slab_rows(U, x0, n).astype(np.float64 if prec == gpu.F64 else np.float32))
    dom.step(nsteps, 0.4)
    torch.cuda.synchronize()
    got, t = slab.solver.download()[:, 2:-2, 2:-2], slab.solver.time()
    want, t1 = run_one(gpu, U, nx, ny, bc, prec, nsteps)
    dom.close()
    assert np.array_equal(got, want)
    assert t == t1
