"""Allocation-free 1D entry point, nest_euler1d_run_noalloc.

Some callers cannot allocate device memory: a host code that owns the whole
GPU through its own memory pool, a plugin host that forbids libraries from
allocating, a real-time loop that must not allocate after start-up.  For them
the library offers one entry point that takes the caller's state buffer and
keeps its own scratch (a second state buffer and the step control block) in a
fixed array inside the library, so the call makes no allocation.

The test calls it through the C ABI twice in a row, each time comparing the
result with the allocating entry points (euler1d_gpu_run / nest_solver_run_to)
under the tolerance every 1D parity test here uses: bit for bit.  The second
call runs on a caller's stream, and a repeat of it must leave the device's
free memory unchanged (no allocation).  It also checks that a size beyond the
array's limit is rejected.  This file is named so that pytest collects it
last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from nest_b200.problems import sod_1d

pytestmark = pytest.mark.gpu
GAMMA = 1.4


def run_noalloc(lib, U, n, h, bc, t_final, cfl, stream=None, free_bytes=None):
    """One call on the caller's device buffer; `stream` a torch stream (None:
    the legacy stream).  free_bytes: a list that receives the device's free
    bytes right before and right after the call."""
    import torch
    state = torch.from_numpy(np.ascontiguousarray(U)).cuda()  # the caller's buffer
    torch.cuda.synchronize()
    steps, t = C.c_int(0), C.c_double(0.0)
    handle = C.c_void_p(stream.cuda_stream) if stream is not None else None
    if free_bytes is not None:
        free_bytes.append(torch.cuda.mem_get_info()[0])
    status = lib.nest_euler1d_run_noalloc(C.c_void_p(state.data_ptr()), n, h, 1.0 / n, GAMMA, bc, t_final,
                                          cfl, C.byref(steps), C.byref(t), handle)
    if free_bytes is not None:
        free_bytes.append(torch.cuda.mem_get_info()[0])
    torch.cuda.synchronize()
    return status, state.cpu().numpy(), steps.value, t.value


def test_noalloc_matches_allocating_entry_points_twice(gpu):
    from nest_b200 import _capi as A
    lib = A.lib

    # call 1: periodic Sod, N = 1024, t = 0.2, CFL 0.4 vs euler1d_gpu_run
    n, h = 1024, 2
    U = sod_1d(n, h)
    status, got, steps, t = run_noalloc(lib, U, n, h, A.BC_PERIODIC, 0.2, 0.4)
    assert status == A.NEST_OK, A.last_error()
    ref = gpu.Euler1DGPU(n, h, 1.0 / n, GAMMA)
    ref.upload(U)
    ref_steps = ref.run(0.2, 0.4)
    want = ref.download()
    assert steps == ref_steps and abs(t - 0.2) < 1e-15
    assert np.array_equal(got[:, h:-h], want[:, h:-h])

    # call 2 (same scratch array, new size and boundary, on a caller's
    # stream): outflow, N = 4099, halo 3, t = 0.1 vs nest_solver_run_to on the
    # tiled path
    import torch
    n, h = 4099, 3
    U = sod_1d(n, h)
    stream = torch.cuda.Stream()
    status, got, steps, t = run_noalloc(lib, U, n, h, A.BC_OUTFLOW, 0.1, 0.4, stream=stream)
    assert status == A.NEST_OK, A.last_error()
    s = gpu.Solver(1, n, halo=h, bc=A.BC_OUTFLOW, flags=A.FLAG_NO_RESIDENT)
    s.upload(U)
    ref_steps = s.run_to(0.1, 0.4)
    want = s.download()
    assert steps == ref_steps and t == s.time()[0]
    assert np.array_equal(got[:, h:-h], want[:, h:-h])

    # the same call again (its kernels are loaded by now): the device's free
    # memory is the same before and after, and so is the result
    free = []
    status, again, steps2, _ = run_noalloc(lib, U, n, h, A.BC_OUTFLOW, 0.1, 0.4, stream=stream, free_bytes=free)
    assert status == A.NEST_OK, A.last_error()
    assert free[0] == free[1], f"free device memory changed across the call: {free}"
    assert steps2 == steps and np.array_equal(again, got)


def test_noalloc_rejects_sizes_beyond_its_array(gpu):
    from nest_b200 import _capi as A
    lib = A.lib
    n = A.NOALLOC_MAX_CELLS  # n + 2h exceeds the limit
    dummy = C.c_double(0.0)
    status = lib.nest_euler1d_run_noalloc(C.byref(dummy), n, 2, 1.0 / n, GAMMA, A.BC_PERIODIC, 0.1, 0.4,
                                          None, None, None)
    assert status == A.NEST_ERR_INVALID
    assert "NEST_NOALLOC_MAX_CELLS" in A.last_error()
