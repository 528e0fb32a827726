"""Device patch halo exchange on nest's per-patch storage, checked against
nest's own tests (tests/test_core.cpp:406-550) and, on random data, against
nest's execute_all_exchanges bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(gpu, x, data):
    import torch
    t = torch.from_numpy(data).cuda()
    x.execute_device(t.data_ptr())
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_plan_structure(gpu):
    # halo_exchange_plan_structure, test_core.cpp:406-424
    x = gpu.PeriodicExchange(1, 12, 3, 1, 1)
    assert list(x.peers[0:2]) == [2, 1]
    assert x.npatch == 3 and list(x.boxes[:, 2]) == [4, 4, 4]


def test_periodic_1d_values(gpu):
    # halo_exchange_periodic_1d_correctness, test_core.cpp:426-458
    x = gpu.PeriodicExchange(1, 12, 3, 1, 1)
    d = np.zeros(x.size)
    for p in range(3):
        x.patch_view(d, p)[0, 1:-1] = p
    d = run(gpu, x, d)
    v = [x.patch_view(d, p)[0] for p in range(3)]
    assert (v[0][0], v[0][-1], v[1][0], v[1][-1], v[2][0], v[2][-1]) == (2, 1, 0, 2, 1, 0)


def test_multivar_and_width2(gpu):
    # halo_exchange_multivar_correctness (460-482) and _wider_halos (484-505)
    x = gpu.PeriodicExchange(1, 8, 2, 3, 1)
    d = np.zeros(x.size)
    for p in range(2):
        v = x.patch_view(d, p)
        v[0, 1:-1], v[1, 1:-1], v[2, 1:-1] = p, p + 10, p + 100
    d = run(gpu, x, d)
    assert list(x.patch_view(d, 0)[:, 0]) == [1.0, 11.0, 101.0]
    x = gpu.PeriodicExchange(1, 20, 2, 1, 2)
    d = np.zeros(x.size)
    for p in range(2):
        s0, _, n0, _ = x.boxes[p]
        x.patch_view(d, p)[0, 2:-2] = np.arange(s0, s0 + n0)
    d = run(gpu, x, d)
    assert list(x.patch_view(d, 0)[0, [0, 1, -2, -1]]) == [18.0, 19.0, 10.0, 11.0]


def test_periodic_2d_faces(gpu):
    # halo_exchange_periodic_2d_faces_correctness, test_core.cpp:507-550
    nx, ny = 6, 4
    x = gpu.PeriodicExchange(2, nx, 2, 1, 1, ny=ny, npy=2)
    d = np.zeros(x.size)
    for p in range(4):
        s0, s1, n0, n1 = x.boxes[p]
        I, J = np.meshgrid(np.arange(s0, s0 + n0), np.arange(s1, s1 + n1), indexing="ij")
        x.patch_view(d, p)[0, 1:-1, 1:-1] = I + 1000 * J
    d = run(gpu, x, d)
    for p in range(4):
        s0, s1, n0, n1 = x.boxes[p]
        v = x.patch_view(d, p)[0]
        for j in range(s1, s1 + n1):
            assert v[0, j - s1 + 1] == (s0 - 1) % nx + 1000 * (j % ny)
            assert v[-1, j - s1 + 1] == (s0 + n0) % nx + 1000 * (j % ny)
        for i in range(s0, s0 + n0):
            assert v[i - s0 + 1, 0] == i % nx + 1000 * ((s1 - 1) % ny)
            assert v[i - s0 + 1, -1] == i % nx + 1000 * ((s1 + n1) % ny)


@pytest.mark.parametrize("dim,nx,ny,npx,npy,nv,h", [(1, 37, 1, 5, 1, 3, 2), (2, 23, 19, 3, 4, 4, 2),
                                                    (2, 64, 64, 4, 4, 4, 2), (2, 10, 9, 2, 3, 1, 1)])
def test_matches_nest_executor(gpu, ref, dim, nx, ny, npx, npy, nv, h):
    import ctypes as C
    x = gpu.PeriodicExchange(dim, nx, npx, nv, h, ny=ny, npy=npy)
    d = np.random.default_rng(nx * ny).standard_normal(x.size)
    want = d.copy()
    dp = C.POINTER(C.c_double)
    if dim == 1:
        ref.L.ref_exchange_1d(want.ctypes.data_as(dp), nx, npx, nv, h)
    else:
        ref.L.ref_exchange_2d(want.ctypes.data_as(dp), nx, ny, npx, npy, nv, h)
    got = run(gpu, x, d)
    assert np.array_equal(got, want)
    got32 = None
    import torch
    t = torch.from_numpy(d.astype(np.float32)).cuda()
    x.execute_device(t.data_ptr(), gpu.F32)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), want.astype(np.float32))
