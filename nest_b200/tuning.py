"""Launch-shape autotuner for the 2D stage kernels.

The tunables are the rows each warp marches per tile and the warps per block
(nest_solver_set_tiling).  A sweep times every candidate with profiled steps
(CUDA events between the stage kernels) on a scratch solver of the requested
size and keeps the fastest.  Results are cached in JSON keyed by
(device name, SM count, form, nx, ny); the cache ships with the package
(tuning_cache.json) and is extended at run time.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

CACHE = Path(os.environ.get("NEST_B200_TUNING", Path(__file__).resolve().parent / "tuning_cache.json"))
ROWS = (16, 24, 32, 64, 128)
WARPS = (1, 2, 4, 8)
DEFAULT = {"f32": (32, 4), "f64": (32, 4)}


def _device_key():
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|{p.multi_processor_count}"


def _load():
    if CACHE.exists():
        try:
            return json.loads(CACHE.read_text())
        except (OSError, json.JSONDecodeError):
            return {}
    return {}


def _key(form, nx, ny):
    return f"{_device_key()}|{form}|{nx}x{ny}"


def sweep(form: str, nx: int, ny: int, steps: int = 6, rows=ROWS, warps=WARPS):
    """Time every (rows, warps) candidate; returns {(rows, warps): ms per step}."""
    import nest_b200 as nb
    from nest_b200.problems import riemann_2d
    prec = nb.F32 if form == "f32" else nb.F64
    U = riemann_2d(nx, ny)
    if form == "f32":
        U = U.astype(np.float32)
    s = nb.Solver(2, nx, ny, bc=nb.BC_OUTFLOW, precision=prec)
    times = {}
    for r in rows:
        for w in warps:
            s.set_tiling(r, w)
            s.upload(U)
            s.step_profiled(2, 0.4)  # warm
            _, _, tot = s.step_profiled(steps, 0.4)
            times[(r, w)] = tot / steps
    s.close()
    return times


def autotune(form: str, nx: int, ny: int, steps: int = 6, save: bool = True):
    times = sweep(form, nx, ny, steps)
    best = min(times, key=times.get)
    if save:
        cache = _load()
        cache[_key(form, nx, ny)] = {"rows_per_tile": best[0], "warps_per_block": best[1],
                                      "ms_per_step": times[best],
                                      "candidates": {f"{r}x{w}": t for (r, w), t in sorted(times.items())}}
        try:
            CACHE.write_text(json.dumps(cache, indent=1, sort_keys=True))
        except OSError:
            pass
    return best, times


def best_tiling(form: str, nx: int, ny: int, tune_if_missing: bool = True):
    """Cached best (rows_per_tile, warps_per_block) for this device, form and
    size; tunes (a few hundred ms) when the cache has no entry."""
    e = _load().get(_key(form, nx, ny))
    if e:
        return int(e["rows_per_tile"]), int(e["warps_per_block"])
    if tune_if_missing:
        best, _ = autotune(form, nx, ny)
        return best
    return DEFAULT[form]


def best_batch_tiling(batch, nx, ny, steps: int = 4, save: bool = True):
    """Cached (rows per item, warps per block, blocks per SM) for a batch of
    these sizes on this device; sweeps the candidates on the batch itself
    (its state is advanced by the sweep: call before uploading)."""
    import hashlib
    key = f"{_device_key()}|batch|{hashlib.sha1(np.asarray([nx, ny]).tobytes()).hexdigest()[:12]}|{len(nx)}"
    cache = _load()
    if key in cache:
        e = cache[key]
        return int(e["rows_per_tile"]), int(e["warps_per_block"]), int(e["blocks_per_sm"])
    times = {}
    for r in (16, 32, 64):
        for w in (1, 2, 4):
            for bps in (0, 4):
                batch.set_tiling(r, w, bps)
                batch.step_profiled(1, 0.4)
                _, _, tot = batch.step_profiled(steps, 0.4)
                times[(r, w, bps)] = tot / steps
    best = min(times, key=times.get)
    if save:
        cache[key] = {"rows_per_tile": best[0], "warps_per_block": best[1], "blocks_per_sm": best[2],
                      "ms_per_step": times[best]}
        try:
            CACHE.write_text(json.dumps(cache, indent=1, sort_keys=True))
        except OSError:
            pass
    return best


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="sweep launch shapes and cache the best")
    ap.add_argument("--sizes", default="4096", help="comma-separated square sizes")
    ap.add_argument("--forms", default="f32,f64")
    ap.add_argument("--out", default="", help="also write the cache to this path")
    a = ap.parse_args()
    for n in [int(x) for x in a.sizes.split(",")]:
        for f in a.forms.split(","):
            best, times = autotune(f, n, n)
            print(f, n, "best", best, "ms/step %.4f" % times[best])
            for k, v in sorted(times.items(), key=lambda kv: kv[1]):
                print("   ", k, "%.4f" % v)
    if a.out:
        Path(a.out).write_text(CACHE.read_text())
