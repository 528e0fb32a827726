"""nest's own callers of its GPU C ABI, compiled unchanged against this
library (tests/dropin/Makefile: nest's tests/test_euler_cuda.cpp and
examples/benchmark/benchmark_euler1d.cpp with NEST_HAS_CUDA, both including
nest's src/backend_cuda/euler1d_solver.hpp and linking libnest_b200.so in
place of nest's CUDA library).

* test_euler_cuda runs nest's CPU solver and the GPU solver on the periodic
  Sod problem (N = 100, t = 0.1, CFL 0.3) and passes when every difference is
  below 1e-8 (tests/test_euler_cuda.cpp:280-306); here the differences are 0.
* benchmark_euler1d times nest's OpenMP CPU loop and then the GPU through
  euler1d_gpu_create / upload / run_timed / download / destroy
  (benchmark_euler1d.cpp:235-257); both take the same number of steps."""
from __future__ import annotations

import os
import re
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
BUILD = ROOT / "tests" / "dropin" / "_build"


def prog(name):
    p = BUILD / name
    if not p.exists():
        pytest.skip(f"{p} not built (make -C tests/dropin REF=<nest tree>)")
    return str(p)


def test_nest_cpu_vs_gpu_test_passes(gpu):
    r = subprocess.run([prog("test_euler_cuda")], capture_output=True, text=True, timeout=300)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out
    assert "PASS: GPU and CPU results match" in out, out
    assert "GPU: 70 steps" in out, out
    diffs = [float(v) for v in re.findall(r"Max difference \(\w+\):\s+(\S+)", out)]
    assert len(diffs) == 3 and max(diffs) == 0.0, out


def test_nest_benchmark_gpu_arm(gpu):
    env = dict(os.environ, OMP_NUM_THREADS=str(len(os.sched_getaffinity(0))))
    r = subprocess.run([prog("benchmark_euler1d"), "4096", "0.05"], capture_output=True, text=True, timeout=600,
                       env=env)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out
    assert "GPU Benchmark (CUDA)" in out and "Error:" not in out, out
    steps = [int(v) for v in re.findall(r"Steps:\s+(\d+)", out)]
    assert len(steps) == 2 and steps[0] == steps[1] > 0, out  # CPU and GPU take the same steps
    assert "Speedup (GPU/CPU)" in out, out
