"""Device pipeline executor (nest_pipeline_*) against nest's own pipeline
executor and its sod1d example.

* nest::execute (include/nest/pipeline.hpp:140-151) of a Reduce stage (dt
  from the CFL rule), an Exchange stage and a Compute stage (euler_rhs_t,
  examples/sod1d/euler1d.hpp:279-397, with its one-sided patch edges), run on
  nest's own patches through oracle/_ref, equals the device pipeline of the
  same stages bit for bit: state and every dt, uneven patches, three
  limiters.
* nest's sod1d time step (examples/sod1d/sod1d.cpp:219-302) as device
  stages, run to t = 0.2 from CUDA graphs, equals the oracle's restatement of
  sod1d bit for bit and nest's own output file to its 11 digits.
* The positivity stage stops a run on nest's schedule (every 10th step)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
G = 1.4


def smooth_sod(n, seed, jump=True):
    """A Sod-like state with smooth perturbations; without the jump (for the
    unlimited reconstruction, which the jump would drive to negative
    pressures) a smooth wave."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    base = np.where(x < 0.5, 1.0, 0.125) if jump else 0.6 + 0.2 * np.cos(2 * np.pi * x)
    rho = base * (1 + 0.05 * np.sin(6 * np.pi * x)) + 0.01 * rng.random(n)
    u = 0.2 * np.sin(2 * np.pi * x)
    p = (np.where(x < 0.5, 1.0, 0.1) if jump else 0.5 + 0.1 * np.sin(2 * np.pi * x)) * (1 + 0.02 * rng.random(n))
    return np.stack([rho, rho * u, p / (G - 1) + 0.5 * rho * u * u])


def device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n,npatch,limiter", [(403, 5, 0), (400, 4, 1), (257, 3, 2)])
def test_matches_nest_execute(gpu, ref, n, npatch, limiter):
    from nest_b200 import pipeline as P
    nexec, cfl = 25, 0.4
    U0 = smooth_sod(n, n, jump=limiter != 2)
    want, want_dts = ref.pipeline_euler1d(U0, npatch, 2, G, cfl, nexec, limiter)
    pipe = P.Pipeline(1, n, npatch, halo=2, limiter=limiter, nwork=1)
    pipe.add(P.CFL_DT, src=P.STATE, param=cfl).add(P.EXCHANGE, src=P.STATE)
    pipe.add(P.EULER_RHS, src=P.STATE, dst=1).add(P.COPY, src=1, dst=P.STATE).add(P.CLOCK)
    d = device(pipe.scatter(U0))
    dts = []
    for _ in range(nexec):
        pipe.execute(d.data_ptr())
        dts.append(pipe.clock()[1])
    got = pipe.gather(d.cpu().numpy())
    assert np.array_equal(np.array(dts), want_dts)
    assert np.array_equal(got, want)
    t, _, steps = pipe.clock()
    assert steps == nexec and t == sum_sequential(want_dts)
    pipe.close()


def sum_sequential(dts):
    t = 0.0
    for d in dts:
        t += d
    return t


def sod1d_oracle(oracle, n=400, npatch=4, h=2, tf=0.2, cfl=0.4):
    """The sod1d example restated on the oracle's patch stage (the same
    restatement tests/test_oracle.py pins against nest's own output)."""
    m = n // npatch
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) * dx
    rho = np.where(x < 0.5, 1.0, 0.125)
    p = np.where(x < 0.5, 1.0, 0.1)
    Ug = np.stack([rho, 0 * rho, p / (G - 1)])

    def patches_of(U):
        return [np.ascontiguousarray(U[:, np.arange(k * m - h, (k + 1) * m + h) % n]) for k in range(npatch)]

    t, steps = 0.0, 0
    while t < tf:
        ms = 0.0
        for i in range(n):
            r, mo, e = Ug[:, i]
            ms = max(ms, abs(mo / r) + math.sqrt(G * oracle.L.orc_pressure(G, r, mo, e) / r))
        dt = min(cfl * dx / ms, tf - t)
        U0 = Ug.copy()
        U1 = np.concatenate([oracle.patch_stage1d(Q, m, h, dx, dt, G)[:, h:-h] for Q in patches_of(Ug)], axis=1)
        U2 = np.concatenate([oracle.patch_stage1d(Q, m, h, dx, dt, G)[:, h:-h] for Q in patches_of(U1)], axis=1)
        Ug = 0.5 * U0 + 0.5 * U2
        t += dt
        steps += 1
    return Ug, t, steps


def test_sod1d_example_on_device(gpu, oracle):
    from nest_b200.pipeline import sod1d_pipeline
    n, npatch = 400, 4
    want, t_want, steps_want = sod1d_oracle(oracle, n, npatch)
    pipe = sod1d_pipeline(n, npatch, cfl=0.4)
    x = (np.arange(n) + 0.5) / n
    rho = np.where(x < 0.5, 1.0, 0.125)
    U0 = np.stack([rho, 0 * rho, np.where(x < 0.5, 1.0, 0.1) / (G - 1)])
    d = device(pipe.scatter(U0))
    steps = pipe.run(d.data_ptr(), 0.2)
    t, _, total = pipe.clock()
    got = pipe.gather(d.cpu().numpy())
    assert steps == total == steps_want and t == t_want
    assert np.array_equal(got, want)
    # nest's own sod_0009.dat (x, rho, u, p with 11 significant digits)
    gold = np.load(GOLDEN / "sod1d_final.npy")
    u = got[1] / got[0]
    pr = np.maximum((G - 1) * (got[2] - 0.5 * got[0] * u * u), 0.0)
    assert np.allclose(got[0], gold[:, 1], rtol=2e-10, atol=0)
    assert np.allclose(u, gold[:, 2], rtol=2e-10, atol=1e-14)
    assert np.allclose(pr, gold[:, 3], rtol=2e-10, atol=0)
    # graph-replayed runs equal single executions (no stopping time to clip dt)
    pipe.set_clock()
    d1 = device(pipe.scatter(U0))
    assert pipe.run(d1.data_ptr(), 1e9, max_steps=48) == 48
    c1 = pipe.clock()
    pipe.set_clock()
    d2 = device(pipe.scatter(U0))
    for _ in range(48):
        pipe.execute(d2.data_ptr())
    # execute() only enqueues on the pipeline's stream; clock() waits for it
    assert pipe.clock() == c1
    assert np.array_equal(d1.cpu().numpy(), d2.cpu().numpy())
    pipe.close()


def test_positivity_stage_stops_on_nests_schedule(gpu):
    from nest_b200.pipeline import sod1d_pipeline
    n, npatch = 400, 4
    x = (np.arange(n) + 0.5) / n
    rho = np.ones(n)
    u = 0.1 * np.sin(2 * np.pi * x)
    U0 = np.stack([rho, rho * u, 1.0 / (G - 1) + 0.5 * rho * u * u])
    # a band of cells moving at u = 2 with E < 1/2 rho u^2 (p < 0): its uniform
    # interior keeps p <= 0, so the check every 10th step finds it at step 10
    U0[1, 100:200], U0[2, 100:200] = 2.0, 0.4
    pipe = sod1d_pipeline(n, npatch, cfl=0.4, check_every=10)
    d = device(pipe.scatter(U0))
    with pytest.raises(gpu.NestError) as ei:
        pipe.run(d.data_ptr(), 0.2)
    msg = str(ei.value)
    assert "NEST_ERR_NUMERIC" in msg and "at step 10 " in msg, msg
    pipe.close()
