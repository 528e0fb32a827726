"""bench.py's reference arm on the CPU: the nest scheme's CPU implementation
(the oracle, OpenMP on the host cores) on a small case of the benchmark
workload prints one JSON line with the keys of the benchmark contract, and
runs without importing the nest_b200 package or loading its CUDA library."""
from __future__ import annotations

import json
import subprocess
import sys

from conftest import ROOT

WRAPPER = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--n", "256", "--steps", "2", "--warmup", "1"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    if e.code not in (None, 0):
        raise
loaded = [m for m in sys.modules if m == "nest_b200" or m.startswith("nest_b200.")]
libs = [l for l in open("/proc/self/maps").read().split() if l.endswith("libnest_b200.so")]
print("LOADED", loaded + libs)
"""


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, "-c", WRAPPER], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "cell-updates/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"] == "riemann2d 256x256 f64" and "fit in L2" in d["config"]["l2"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    loaded = [l for l in out.stdout.splitlines() if l.startswith("LOADED")]
    assert loaded == ["LOADED []"], loaded


def test_reference_arm_under_torchrun():
    """Launched like the CUDA arm at N = 2 (torchrun, one process per rank):
    rank 0 alone prints one line, for the same (2 n) x n workload the CUDA arm
    runs at that world size; the other rank exits 0 without work."""
    import random
    port = random.randint(29100, 29900)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--size", "256", "--steps", "2", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["config"]["workload"] == "riemann2d 512x256 f64" and d["config"]["nx"] == 512
    assert "512x256" in d["cpu_baseline"]["sample"]
