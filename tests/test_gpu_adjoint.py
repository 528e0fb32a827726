"""Discrete adjoint of the 1D FP64 solver (periodic, dt frozen): gradients
against central finite differences on random directions, uniform vs binomial
checkpointing, and the torch.autograd wrapper."""
from __future__ import annotations

import numpy as np
import pytest

from nest_b200.problems import fourier_fields_1d, prim_to_cons_1d

pytestmark = pytest.mark.gpu
G = 1.4


def loss_and_lam(gpu, U0, target_rho, n, nsteps, dts):
    """L = 1/2 sum (rho_T - target)^2 dx with the forward run on frozen dts."""
    s = gpu.Solver(1, n, bc=gpu.BC_PERIODIC, flags=gpu.FLAG_NO_RESIDENT)
    s.freeze_dts(dts)
    s.upload(U0)
    s.step(nsteps, 0.4)
    UT = s.download()
    r = UT[0, 2:-2] - target_rho
    return 0.5 * np.sum(r * r) / n


@pytest.mark.parametrize("policy,param", [(0, 16), (1, 6)])
def test_adjoint_matches_finite_differences(gpu, policy, param):
    from nest_b200.adjoint import Adjoint
    n, nsteps = 256, 120
    U0 = prim_to_cons_1d(*fourier_fields_1d(n, seed=1))
    tgt = prim_to_cons_1d(*fourier_fields_1d(n, seed=2))[0, 2:-2]
    s = gpu.Solver(1, n, bc=gpu.BC_PERIODIC, flags=gpu.FLAG_NO_RESIDENT)
    s.upload(U0)
    adj = Adjoint(s, nsteps, policy, param)
    adj.forward(0.4)
    dts = adj.dts()
    UT = s.download()
    lamT = np.zeros_like(UT)
    lamT[0, 2:-2] = (UT[0, 2:-2] - tgt) / n
    lam0 = adj.backward(lamT)
    rng = np.random.default_rng(5)
    x = (np.arange(n) + 0.5) / n
    for _ in range(6):
        d = np.zeros_like(U0)
        for k in range(3):
            c = rng.standard_normal(4)
            d[k, 2:-2] = sum(c[m] * np.sin(2 * np.pi * (m + 1) * x + c[(m + 1) % 4]) for m in range(4))
        # central FD; a small step keeps the +-eps pair on the same side of the
        # scheme's minmod / HLLE branch kinks (a crossed kink biases FD, not the adjoint)
        eps = 1e-8
        fd = (loss_and_lam(gpu, U0 + eps * d, tgt, n, nsteps, dts) -
              loss_and_lam(gpu, U0 - eps * d, tgt, n, nsteps, dts)) / (2 * eps)
        ad = float(np.sum(lam0[:, 2:-2] * d[:, 2:-2]))
        assert abs(ad - fd) <= 1e-6 * abs(fd) + 1e-14, (ad, fd)


def test_adjoint_equals_exact_tangent(gpu):
    """Exact check: the adjoint's directional derivative equals the
    tangent-linear model (dual numbers through the oracle's stage, same
    branches as the forward) to rounding."""
    from oracle.tangent import tangent_rollout
    from nest_b200.adjoint import Adjoint
    n, nsteps = 48, 12
    U0 = prim_to_cons_1d(*fourier_fields_1d(n, seed=7))
    s = gpu.Solver(1, n, bc=gpu.BC_PERIODIC, flags=gpu.FLAG_NO_RESIDENT)
    s.upload(U0)
    adj = Adjoint(s, nsteps, 0, 5)
    adj.forward(0.4)
    dts = adj.dts()
    UT = s.download()
    rng = np.random.default_rng(11)
    w = rng.standard_normal((3, n))           # loss L = w . U_T
    lamT = np.zeros_like(UT)
    lamT[:, 2:-2] = w
    lam0 = adj.backward(lamT)
    for _ in range(3):
        d = rng.standard_normal((3, n))
        UTt, dUT = tangent_rollout(U0[:, 2:-2], d, dts, 1.0 / n)
        assert np.array_equal(np.array(UTt), UT[:, 2:-2])  # same trajectory as the GPU
        jvp = float(np.sum(w * np.array(dUT)))
        vjp = float(np.sum(lam0[:, 2:-2] * d))
        assert abs(jvp - vjp) <= 1e-11 * max(1.0, abs(jvp)), (jvp, vjp)
    adj.close()
    s.close()


def test_uniform_and_binomial_agree(gpu):
    from nest_b200.adjoint import Adjoint
    n, nsteps = 512, 97
    U0 = prim_to_cons_1d(*fourier_fields_1d(n, seed=3))
    lamT = np.zeros_like(U0)
    lamT[:, 2:-2] = np.random.default_rng(1).standard_normal((3, n))
    outs = []
    for policy, param in [(0, 10), (0, 97), (1, 4), (1, 30)]:
        s = gpu.Solver(1, n, bc=gpu.BC_PERIODIC, flags=gpu.FLAG_NO_RESIDENT)
        s.upload(U0)
        adj = Adjoint(s, nsteps, policy, param)
        adj.forward(0.4)
        outs.append(adj.backward(lamT))
        st = adj.stats()
        assert st["recomputed_steps"] >= 0 and st["checkpoint_bytes"] > 0
    for o in outs[1:]:
        assert np.array_equal(o[:, 2:-2], outs[0][:, 2:-2])


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_uniform_and_binomial_agree_2d(gpu, prec):
    """2D adjoint under the uniform schedule and under binomial schedules
    with few and many snapshots (re-advances that start from a snapshot in
    place and end in the next one): the same gradient bit for bit."""
    from nest_b200.adjoint import Adjoint
    from nest_b200.problems import kelvin_helmholtz
    nx, ny, nsteps = 64, 48, 37
    dt = np.float64 if prec == "f64" else np.float32
    p = gpu.F64 if prec == "f64" else gpu.F32
    U0 = kelvin_helmholtz(nx, ny, seed=2).astype(dt)
    lamT = np.zeros(U0.shape, dtype=dt)
    lamT[:, 2:-2, 2:-2] = np.random.default_rng(4).standard_normal((4, nx, ny))
    outs = []
    for policy, param in [(0, 10), (1, 3), (1, 9), (1, 37)]:
        s = gpu.Solver(2, nx, ny, bc=gpu.BC_PERIODIC, precision=p)
        s.upload(U0)
        adj = Adjoint(s, nsteps, policy, param)
        adj.forward(0.4)
        outs.append(adj.backward(lamT))
    for o in outs[1:]:
        assert np.array_equal(o[:, 2:-2, 2:-2], outs[0][:, 2:-2, 2:-2])


def test_autograd_rollout(gpu):
    import torch
    from nest_b200.adjoint import rollout_1d
    n, nsteps = 128, 40
    rho, u, p = (torch.tensor(f, device="cuda", requires_grad=True) for f in fourier_fields_1d(n, seed=4))
    U0 = torch.stack([rho, rho * u, p / (G - 1.0) + 0.5 * rho * u * u])
    UT = rollout_1d(U0, nsteps, cfl=0.4, policy=0, param=8)
    loss = 0.5 * (UT[0] ** 2).sum() / n
    loss.backward()
    assert rho.grad is not None and torch.isfinite(rho.grad).all() and torch.isfinite(p.grad).all()
    # check one directional derivative in primitive space by FD (dts frozen)
    from nest_b200.adjoint import Adjoint
    W = [x.detach().cpu().numpy() for x in (rho, u, p)]
    s = gpu.Solver(1, n, bc=gpu.BC_PERIODIC, flags=gpu.FLAG_NO_RESIDENT)
    s.upload(prim_to_cons_1d(*W))
    a = Adjoint(s, nsteps, 0, 8)
    a.forward(0.4)
    dts = a.dts()
    dr = np.cos(2 * np.pi * 3 * (np.arange(n) + 0.5) / n)

    def L(eps):
        s2 = gpu.Solver(1, n, bc=gpu.BC_PERIODIC, flags=gpu.FLAG_NO_RESIDENT)
        s2.freeze_dts(dts)
        s2.upload(prim_to_cons_1d(W[0] + eps * dr, W[1], W[2]))
        s2.step(nsteps, 0.4)
        return 0.5 * np.sum(s2.download()[0, 2:-2] ** 2) / n

    fd = (L(1e-6) - L(-1e-6)) / 2e-6
    ad = float(np.sum(rho.grad.cpu().numpy() * dr))
    assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)


def adjoint2d_case(gpu, nx, ny, nsteps, prec, seed=3, policy=0, param=8, smooth=False):
    from nest_b200.adjoint import Adjoint
    from nest_b200.problems import fourier_fields_2d, kelvin_helmholtz
    U0 = fourier_fields_2d(nx, ny, seed) if smooth else kelvin_helmholtz(nx, ny, seed=seed)
    dt = np.float64 if prec == gpu.F64 else np.float32
    s = gpu.Solver(2, nx, ny, bc=gpu.BC_PERIODIC, precision=prec)
    s.upload(U0.astype(dt))
    adj = Adjoint(s, nsteps, policy, param)
    adj.forward(0.4)
    return U0, s, adj


def test_adjoint2d_equals_exact_tangent(gpu):
    from oracle.tangent import tangent_rollout_2d
    nx, ny, nsteps = 12, 10, 3
    U0, s, adj = adjoint2d_case(gpu, nx, ny, nsteps, gpu.F64)
    dts = adj.dts()
    UT = s.download()
    rng = np.random.default_rng(2)
    w = rng.standard_normal((4, nx, ny))
    lamT = np.zeros_like(UT)
    lamT[:, 2:-2, 2:-2] = w
    lam0 = adj.backward(lamT)
    for _ in range(2):
        d = rng.standard_normal((4, nx, ny))
        val, der = tangent_rollout_2d(U0[:, 2:-2, 2:-2], d, dts, 1.0 / nx, 1.0 / ny)
        assert np.array_equal(np.array(val), UT[:, 2:-2, 2:-2])
        jvp = float(np.sum(w * np.array(der)))
        vjp = float(np.sum(lam0[:, 2:-2, 2:-2] * d))
        assert abs(jvp - vjp) <= 1e-11 * max(1.0, abs(jvp)), (jvp, vjp)


def ke_v_loss_and_lambda(U, nx, ny):
    """L = integral of 1/2 rho v^2 dA and its gradient w.r.t. (rho, mu, mv, E)."""
    r, mv = U[0, 2:-2, 2:-2].astype(np.float64), U[2, 2:-2, 2:-2].astype(np.float64)
    v = mv / r
    dA = 1.0 / (nx * ny)
    lam = np.zeros(U.shape)
    lam[0, 2:-2, 2:-2] = -0.5 * v * v * dA
    lam[2, 2:-2, 2:-2] = v * dA
    return 0.5 * np.sum(r * v * v) * dA, lam


def test_adjoint2d_finite_differences_fp64(gpu):
    """Central differences against the adjoint on a smooth state.  The KH
    state has exactly uniform bands where the limiter sits at minmod(0, 0):
    there the scheme is only piecewise linear and a difference quotient
    measures a one-sided derivative the subgradient does not (the exact
    tangent test covers KH)."""
    nx, ny, nsteps = 48, 40, 30
    U0, s, adj = adjoint2d_case(gpu, nx, ny, nsteps, gpu.F64, seed=4, smooth=True)
    dts = adj.dts()
    L0, lamT = ke_v_loss_and_lambda(s.download(), nx, ny)
    lam0 = adj.backward(lamT)
    rng = np.random.default_rng(8)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")

    def L(U):
        s2 = gpu.Solver(2, nx, ny, bc=gpu.BC_PERIODIC, precision=gpu.F64)
        s2.freeze_dts(dts)
        s2.upload(U)
        s2.step(nsteps, 0.4)
        return ke_v_loss_and_lambda(s2.download(), nx, ny)[0]

    for _ in range(4):
        d = np.zeros_like(U0)
        for k in range(4):
            a, b, c = rng.standard_normal(3)
            d[k, 2:-2, 2:-2] = a * np.sin(2 * np.pi * (X + b)) * np.cos(2 * np.pi * (2 * Y + c))
        eps = 1e-8
        fd = (L(U0 + eps * d) - L(U0 - eps * d)) / (2 * eps)
        ad = float(np.sum(lam0[:, 2:-2, 2:-2] * d[:, 2:-2, 2:-2]))
        assert abs(ad - fd) <= 1e-6 * abs(fd) + 1e-15, (ad, fd)


def test_adjoint2d_fp32_vs_fp64(gpu):
    """Gradient of the v kinetic energy w.r.t. the initial v field: FP32
    forward + adjoint against the FP64 adjoint (binomial checkpointing)."""
    nx = ny = 64
    out = {}
    for prec in (gpu.F64, gpu.F32):
        U0, s, adj = adjoint2d_case(gpu, nx, ny, 40, prec, seed=5, policy=1, param=6)
        _, lamT = ke_v_loss_and_lambda(s.download(), nx, ny)
        lam0 = adj.backward(lamT).astype(np.float64)
        r0 = U0[0, 2:-2, 2:-2]
        v0 = U0[2, 2:-2, 2:-2] / r0
        out[prec] = lam0[2, 2:-2, 2:-2] * r0 + lam0[3, 2:-2, 2:-2] * r0 * v0  # dL/dv0
    g64, g32 = out[gpu.F64], out[gpu.F32]
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    assert rel < 1e-3, rel


@pytest.mark.parametrize("nx,ny", [(12, 10), (48, 40), (130, 118), (70, 64), (200, 232)])
def test_adjoint2d_fp32_row_march(gpu, nx, ny, monkeypatch):
    """The FP32 form's adjoint stage, a packed row march with one strip of
    56 columns per warp (several strips, ragged strips and row segments,
    domains narrower than a strip), against the FP32 tile kernel on the same
    FP32 trajectory (NEST_ADJOINT2D_TILE=1): smooth fields, 6 steps, random
    final adjoint.  Both reverse the same discrete map; they differ by FP32
    rounding of the reverse sweep (relative L2 about 1e-6).  Against the FP64
    adjoint the difference is larger (1e-3 at 130 x 118): FP32 rounding of
    the trajectory moves a few near-ties of |d1| and |d2| to the other minmod
    branch, which changes that cell's derivative by order one."""
    lam = {}
    for key, tile in (("march", "0"), ("tile", "1")):
        monkeypatch.setenv("NEST_ADJOINT2D_TILE", tile)
        U0, s, adj = adjoint2d_case(gpu, nx, ny, 6, gpu.F32, seed=6, smooth=True)
        UT = s.download()
        w = np.random.default_rng(9).standard_normal((4, nx, ny))
        lamT = np.zeros(UT.shape, dtype=np.float32)
        lamT[:, 2:-2, 2:-2] = w
        lam[key] = adj.backward(lamT).astype(np.float64)[:, 2:-2, 2:-2]
    assert np.all(np.isfinite(lam["march"]))
    rel = np.linalg.norm(lam["march"] - lam["tile"]) / np.linalg.norm(lam["tile"])
    assert rel < 1e-4, rel


@pytest.mark.parametrize("nx,ny", [(64, 63), (40, 27)])
def test_adjoint2d_fp32_odd_ny(gpu, nx, ny):
    """FP32 with an odd ny (the packed row march needs adjacent column pairs,
    so these domains take the tile kernel) against the FP64 adjoint: smooth
    fields, 6 steps; the two differ by FP32 rounding and the few limiter
    branches it moves (a few 1e-4)."""
    lam = {}
    for prec in (gpu.F64, gpu.F32):
        U0, s, adj = adjoint2d_case(gpu, nx, ny, 6, prec, seed=6, smooth=True)
        UT = s.download()
        w = np.random.default_rng(9).standard_normal((4, nx, ny))
        lamT = np.zeros(UT.shape, dtype=UT.dtype)
        lamT[:, 2:-2, 2:-2] = w
        lam[prec] = adj.backward(lamT).astype(np.float64)[:, 2:-2, 2:-2]
    rel = np.linalg.norm(lam[gpu.F32] - lam[gpu.F64]) / np.linalg.norm(lam[gpu.F64])
    assert rel < 5e-3, rel


@pytest.mark.parametrize("nx,ny", [(12, 10), (48, 40), (130, 118), (64, 63), (31, 77)])
def test_adjoint2d_fp64_row_march(gpu, nx, ny, monkeypatch):
    """The FP64 row-march adjoint stage (one column per lane, strips of 26
    columns; odd and narrow domains) against the FP64 tile kernel on the
    same trajectory, smooth fields: same map, same subgradients, FP64
    rounding of the reverse sweep only.  The exact-tangent and
    finite-difference tests above run the row march on KH and smooth data."""
    lam = {}
    for key, tile in (("march", "0"), ("tile", "1")):
        monkeypatch.setenv("NEST_ADJOINT2D_TILE", tile)
        U0, s, adj = adjoint2d_case(gpu, nx, ny, 5, gpu.F64, seed=7, smooth=True)
        UT = s.download()
        w = np.random.default_rng(11).standard_normal((4, nx, ny))
        lamT = np.zeros(UT.shape)
        lamT[:, 2:-2, 2:-2] = w
        lam[key] = adj.backward(lamT)[:, 2:-2, 2:-2]
    rel = np.linalg.norm(lam["march"] - lam["tile"]) / np.linalg.norm(lam["tile"])
    assert rel < 1e-12, rel


def test_adjoint1d_fp32_vs_fp64(gpu):
    """1D adjoint of the FP32 form (FP32 forward, FP32 reverse stages, FP64
    dt sequence) against the FP64 adjoint on the same loss: the L2 misfit
    of the final density, gradient with respect to the initial state."""
    from nest_b200.adjoint import Adjoint
    n, nsteps = 512, 160
    U0 = prim_to_cons_1d(*fourier_fields_1d(n, seed=1))
    tgt = prim_to_cons_1d(*fourier_fields_1d(n, seed=2))[0, 2:-2]
    grads = {}
    for prec, dt in ((gpu.F64, np.float64), (gpu.F32, np.float32)):
        flags = gpu.FLAG_NO_RESIDENT if prec == gpu.F64 else 0
        s = gpu.Solver(1, n, bc=gpu.BC_PERIODIC, precision=prec, flags=flags)
        s.upload(U0.astype(dt))
        adj = Adjoint(s, nsteps, 1, 8)
        adj.forward(0.4)
        UT = s.download().astype(np.float64)
        lamT = np.zeros_like(UT)
        lamT[0, 2:-2] = (UT[0, 2:-2] - tgt) / n
        grads[prec] = adj.backward(lamT.astype(dt)).astype(np.float64)[:, 2:-2]
        adj.close()
        s.close()
    g64, g32 = grads[gpu.F64], grads[gpu.F32]
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    assert np.all(np.isfinite(g32)) and rel < 1e-3, rel


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_autograd_rollout_2d(gpu, prec):
    """rollout_2d (torch.autograd.Function over the 2D adjoint): the gradient
    of a torch loss of U_T w.r.t. the initial v perturbation equals the
    Adjoint API's bit for bit (same snapshots, same kernels), and in FP64 a
    finite difference of the loss (dts frozen) to 1e-6."""
    import torch
    from nest_b200.adjoint import BINOMIAL, Adjoint, rollout_2d
    from nest_b200.problems import fourier_fields_2d
    nx, ny, nsteps = 48, 40, 30
    tdt = torch.float64 if prec == "f64" else torch.float32
    U0np = fourier_fields_2d(nx, ny, 4)[:, 2:-2, 2:-2]
    base = torch.tensor(U0np, dtype=torch.float64, device="cuda")
    dv = torch.zeros((nx, ny), dtype=torch.float64, device="cuda", requires_grad=True)
    rho = base[0]
    U0 = torch.stack([base[0], base[1], base[2] + rho * dv, base[3] + base[2] * dv]).to(tdt)
    UT = rollout_2d(U0, nsteps, cfl=0.4, policy=BINOMIAL, param=6)
    v = UT[2].double() / UT[0].double()
    loss = 0.5 * (UT[0].double() * v * v).sum() / (nx * ny)
    loss.backward()
    g = dv.grad.cpu().numpy()
    assert np.all(np.isfinite(g)) and np.abs(g).max() > 0
    # the same gradient through the Adjoint API
    s = gpu.Solver(2, nx, ny, bc=gpu.BC_PERIODIC, precision=gpu.F64 if prec == "f64" else gpu.F32)
    Uext = np.zeros((4, nx + 4, ny + 4))
    Uext[:, 2:-2, 2:-2] = U0.detach().double().cpu().numpy()
    s.upload(Uext.astype(np.float64 if prec == "f64" else np.float32))
    a = Adjoint(s, nsteps, BINOMIAL, 6)
    a.forward(0.4)
    L0, lamT = ke_v_loss_and_lambda(s.download(), nx, ny)
    lam0 = a.backward(lamT.astype(np.float64 if prec == "f64" else np.float32)).astype(np.float64)
    want = lam0[2, 2:-2, 2:-2] * U0np[0] + lam0[3, 2:-2, 2:-2] * U0np[2]
    tol = 1e-10 if prec == "f64" else 1e-5
    assert np.allclose(g, want, rtol=tol, atol=tol * np.abs(want).max())
    if prec == "f64":
        dts = a.dts()
        x = (np.arange(nx) + 0.5) / nx
        d = np.outer(np.sin(2 * np.pi * x), np.cos(4 * np.pi * (np.arange(ny) + 0.5) / ny))

        def L(eps):
            U = U0np.copy()
            U[3] = U0np[3] + U0np[2] * eps * d + 0.5 * U0np[0] * (eps * d) ** 2
            U[2] = U0np[2] + U0np[0] * eps * d
            s2 = gpu.Solver(2, nx, ny, bc=gpu.BC_PERIODIC, precision=gpu.F64)
            s2.freeze_dts(dts)
            s2.upload(U, gpu.LAYOUT_INTERIOR)
            s2.step(nsteps, 0.4)
            return ke_v_loss_and_lambda(s2.download(), nx, ny)[0]

        fd = (L(1e-7) - L(-1e-7)) / 2e-7
        ad = float(np.sum(g * d))
        assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)


def test_config5_fp32_gradient_tracks_fp64(gpu):
    """The config-5 problem itself (Kelvin-Helmholtz, 2048^2 periodic, 4000
    steps, binomial snapshots in 40 GB, loss = integral of 1/2 rho v^2 dA,
    gradient with respect to the initial v): the FP32 adjoint's gradient stays
    within 5 % (relative L2) of the FP64 adjoint's.  Before the FP32 reverse
    kernels split the minmod slope adjoint at near-ties decided by FP32
    rounding, it was 12.8 here (cosine 0.08)."""
    import bench
    from nest_b200.problems import kelvin_helmholtz
    n, K = 2048, 4000
    U0 = kelvin_helmholtz(n, n, seed=1)
    g64, _, _ = bench.kh_grad_v(U0, n, K, np.float64)
    g32, _, _ = bench.kh_grad_v(U0, n, K, np.float32)
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    cos = np.sum(g32 * g64) / (np.linalg.norm(g32) * np.linalg.norm(g64))
    assert rel < 0.05 and cos > 0.999, (rel, cos)
