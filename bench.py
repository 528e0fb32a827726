"""Benchmark of the nest hot path on B200 (one JSON line on rank 0).

Workload (default, --workload riemann2d): the 2D Euler Riemann problem on
[0,1]^2 with 4096 x 4096 cells (16 x 16 patches of 256^2), outflow
boundaries, CFL 0.4, gamma 1.4, 200 RK2 steps.  A bench step is one RK2 step
of the whole grid (dt reduction, ghost fill, two fused stages).  Metric:
cell-updates/s = interior cells x steps x 2 RK stages
(examples/benchmark/benchmark_euler1d.cpp:217-218).  The headline form is the
plain FP64 form, the arithmetic of the CPU path it is compared with (its
result is checked against that CPU path cell for cell in the same run); the
FP32 form (reconstruction, Riemann solve and update in FP32; FP64 totals,
time, dt and positivity repair) and the plain FP32 form are measured in the
same run under `forms`.

Arms
  --impl ours       (default) the CUDA library through its C ABI.
  --impl reference  the CPU implementation of the same scheme on the host
                    cores (the oracle port: nest has no 2D RK2), one bounded
                    sample per step, FP64.  Rank 0 only.  It loads neither
                    the nest_b200 package nor its library.

Multi-GPU (torchrun, N ranks): one domain of (N*4096) x 4096 cells cut into
N x-slabs of 4096 x 4096, one per GPU (weak scaling): every step max-reduces
the two wave-speed words over NCCL and swaps two ghost rows with each
neighbour before each stage (nest_b200/shard.py).  Timing is the max over
ranks; value counts every rank's cells.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s & %HBM roofline, FP32-batched vs FP64 plain; adjoint/fwd cost"
UNIT = "cell-updates/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["riemann2d"], default="riemann2d")
    ap.add_argument("--n", "--size", dest="n", type=int, default=4096,
                    help="cells per axis (--size under torchrun, whose parser takes --n for its own options)")
    ap.add_argument("--forms", default="f64,f32,f32plain",
                    help="forms to time (f64: the plain FP64 form; f32: FP32 with FP64 totals and repair; "
                         "f32plain: FP32 without them); the first is the headline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--tiling", default="", help="rows,warps: fixed launch shape instead of the tuned one")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched-KH and adjoint measurements")
    ap.add_argument("--slab-path", action="store_true",
                    help="drive the domain through the x-slab driver even on one GPU (a one-rank group)")
    ap.add_argument("--native-slabs", action="store_true",
                    help="x-slabs stepped by the C++ NCCL driver (nest_slab_step, graph-replayed) instead of "
                         "the per-step torch.distributed loop")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=500)
    ap.add_argument("--adjoint-n", type=int, default=65536)
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    ap.add_argument("--fd-directions", type=int, default=32)
    ap.add_argument("--adjoint2d-n", type=int, default=2048)
    ap.add_argument("--adjoint2d-steps", type=int, default=4000)
    ap.add_argument("--no-adjoint2d", action="store_true")
    ap.add_argument("--adjoint2d-horizons", default="500,1000,2000,4000",
                    help="horizons of the adjoint2d_study extra (FP32 and rounded-IC FP64 gradients vs FP64)")
    ap.add_argument("--extras", default="batched,adjoint1d,sod1d,adjoint2d",
                    help="comma list of extra measurements to run (with extras on)")
    return ap.parse_args()


L2_MB = 126  # B200 L2 cache, MB

FORM_TEXT = {"f32": "FP32 state and arithmetic; FP64 conserved totals every step, FP64 time and dt, FP64 "
                     "positivity repair",
             "f32plain": "FP32 state and arithmetic; FP64 time and dt",
             "f64": "plain FP64 form (bit for bit with the CPU oracle)"}


def workload_config(n: int, ws: int, head: str, slab: bool) -> dict:
    """`config` of the JSON line, the same keys for both arms."""
    mb = 4 * (n + 4) ** 2 * (4 if head.startswith("f32") else 8) / 1e6
    return {"workload": f"riemann2d {ws * n}x{n} {head}", "nx": ws * n, "ny": n, "form": FORM_TEXT[head],
            "patches": f"{n // 256}x{n // 256} of 256^2" if n % 256 == 0 else "one",
            "bc": "outflow", "cfl": 0.4, "gamma": 1.4,
            "parallelism": "one GPU" if ws == 1 and not slab else
            f"{ws} x-slabs of {n}x{n} (NCCL halo rows + wave-speed all-reduce)",
            "l2": ("inputs larger than L2 (two state buffers of %.0f MB each)" if mb > L2_MB else
                   "inputs fit in L2 (two state buffers of %.1f MB each): a small case, not the benchmark "
                   "workload") % mb}


def load_problems():
    """nest_b200/problems.py loaded by path (numpy only): the reference arm
    builds its inputs without importing the nest_b200 package, whose import
    loads the CUDA library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_bench_problems", ROOT / "nest_b200" / "problems.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

def dist_setup(force: bool = False):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1 or force:
        if ws == 1:
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
            os.environ.setdefault("MASTER_PORT", "29531")
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allsum(ws, x: float) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def allmax(ws, x: float) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self.proc = None

    def start(self):
        import torch
        ident = str(self.dev)
        try:
            pr = torch.cuda.get_device_properties(self.dev)
            ident = "%08X:%02X:%02X.0" % (int(pr.pci_domain_id), int(pr.pci_bus_id), int(pr.pci_device_id))
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            if vis and vis.split(",")[self.dev].strip().isdigit():
                ident = vis.split(",")[self.dev].strip()
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", ident, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), line.strip()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0: float, t1: float):
        if not self.rows:
            return None
        sel = [r for (t, r) in self.rows if t0 - 0.3 <= t <= t1 + 0.3] or [r for _, r in self.rows]
        mhz, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in sel:
            parts = [p.strip() for p in r.split(",")]
            if len(parts) < 7:
                continue
            try:
                mhz.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not mhz:
            return None
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(mhz)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def alg_bytes_per_cell(form: str):
    """Algorithmic HBM bytes per cell of one launch: stage 1 reads U^n and
    writes U1 (8 values); stage 2 reads U1 and U^n and writes U^{n+1}
    (12 values).  Per cell-update that is 2.5 * 4 vars * s bytes."""
    s = 4 if form.startswith("f32") else 8
    return {"stage1": 8 * s, "stage2": 12 * s, "per_cell_update": 10 * s}


def form_args(form: str):
    """(precision, solver flags) of a timed form: `f32` is the FP32 form with
    FP64 conserved totals every step and FP64 positivity repair, `f32plain`
    the same arithmetic without them, `f64` the plain FP64 form."""
    import nest_b200 as nb
    return {"f32": (nb.F32, nb.FLAG_TOTALS | nb.FLAG_REPAIR), "f32plain": (nb.F32, 0),
            "f64": (nb.F64, 0)}[form]


def tune_form(form: str) -> str:
    return "f32" if form.startswith("f32") else "f64"


def kernel_name(form: str, stage: str) -> str:
    """Name of the stage kernel the bench's form launches (no repair flag)."""
    if form == "f32":  # FP64 repair; FP64 totals in stage 2
        return "k2d_f32x2<1, true, false>" if stage == "stage1" else "k2d_f32x2<2, true, true>"
    if form == "f32plain":
        return f"k2d_f32x2<{stage[-1]}, false, false>"
    return f"k2d_f64r<{stage[-1]}, 0, 0>"  # minmod instance


def traffic_from_profiles(form: str, n: int):
    f = ROOT / "profiles" / "traffic.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text())
    key = f"riemann2d_{form}"
    if key not in d:
        return None
    e = d[key]
    return {k: v * (n * n) / float(e["cells"]) for k, v in e["bytes_per_launch"].items()}


def run_slabs(args, ws, rank, form, cfl, st):
    """N>1: this rank's x-slab of the (ws*n) x n domain.  Returns the timed
    figures of one form (same keys as the one-domain path)."""
    import torch
    import torch.distributed as dist
    import nest_b200 as nb
    from nest_b200.problems import riemann_2d
    from nest_b200.shard import gpu_domain
    from nest_b200.tuning import best_tiling
    n = args.n
    prec, flags = form_args(form)
    dom, ranges = gpu_domain(ws * n, n, bc=nb.BC_OUTFLOW, precision=prec, flags=flags, group=dist.group.WORLD,
                             native=args.native_slabs)
    (slab,), ((x0, nl),) = dom.slabs, ranges
    U = riemann_2d(ws * n, n, rows=(x0, nl))
    U = U.astype(np.float32) if prec == nb.F32 else U
    tiling = tuple(int(v) for v in args.tiling.split(",")) if args.tiling else best_tiling(tune_form(form), nl, n)
    slab.solver.set_tiling(*tiling)
    sst = slab.stream_obj
    slab.solver.upload(U)
    dom.step(args.warmup, cfl)
    slab.solver.sync()
    slab.solver.upload(U)
    slab.solver.reset_time()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.time()
    e0.record(sst)
    dom.step(args.steps, cfl)
    e1.record(sst)
    e1.synchronize()
    t1 = time.time()
    barrier(ws)
    ms = allmax(ws, e0.elapsed_time(e1)) / args.steps
    tsim, nst = slab.solver.time()
    # per-kernel durations: the same steps again with events around each stage
    slab.solver.upload(U)
    slab.solver.reset_time()
    if args.native_slabs:
        # the stage kernels alone (their durations do not depend on the exchanges)
        k1, k2, _ = slab.solver.step_profiled(args.steps, cfl)
    else:
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
        with slab.stream():
            for k in range(args.steps):
                dom.reduce_speeds()
                dom.exchange(0)
                ev[k][0].record(sst)
                slab.stage(1, cfl, 0.0)
                ev[k][1].record(sst)
                dom.exchange(1)
                ev[k][2].record(sst)
                slab.stage(2, cfl, 0.0)
                ev[k][3].record(sst)
        sst.synchronize()
        k1 = [e[0].elapsed_time(e[1]) for e in ev]
        k2 = [e[2].elapsed_time(e[3]) for e in ev]
    out = {"ms": ms, "k1": k1, "k2": k2, "tsim": tsim, "steps": nst, "tiling": tiling, "window": (t0, t1),
           "cells_local": nl * n, "graph_ms": None}
    if not args.no_e2e:
        tdt = torch.float32 if prec == nb.F32 else torch.float64
        hin = torch.empty(U.shape, dtype=tdt, pin_memory=True)
        hin.numpy()[...] = U
        hout = torch.empty(U.shape, dtype=tdt, pin_memory=True)
        barrier(ws)
        torch.cuda.synchronize()
        e0.record(sst)
        nb.solver.check(nb._capi.lib.nest_solver_upload(slab.solver._h, hin.data_ptr(), nb.LAYOUT_EXTENDED), "upload")
        slab.solver.reset_time()
        dom.step(args.steps, cfl)
        nb.solver.check(nb._capi.lib.nest_solver_download(slab.solver._h, hout.data_ptr(), nb.LAYOUT_EXTENDED),
                        "download")
        slab.solver.time()
        e1.record(sst)
        e1.synchronize()
        ems = allmax(ws, e0.elapsed_time(e1))
        out["e2e"] = {"value": ws * nl * n * 2 * args.steps / (ems * 1e-3), "unit": UNIT, "ms_total": ems,
                      "h2d_bytes_per_step": U.nbytes / args.steps, "d2h_bytes_per_step": (U.nbytes + 32) / args.steps,
                      "api": "nest_solver_upload -> SlabDomain.step -> nest_solver_download -> nest_solver_time"}
    barrier(ws)
    torch.cuda.synchronize()
    if args.native_slabs:
        dom.close()  # graphs holding NCCL calls go before the communicator
    else:
        for sl in dom.slabs:
            sl.solver.close()
    return out


def run_ours(args, ws, rank, local):
    import torch
    import nest_b200 as nb
    from nest_b200.problems import riemann_2d
    from nest_b200.tuning import best_tiling

    torch.cuda.set_device(local)
    n = args.n
    cells = n * n
    cfl = 0.4
    hbm, peak_kind = peaks()
    st = torch.cuda.Stream()
    U64 = riemann_2d(n, n) if ws == 1 and not args.slab_path else None
    results = {}
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    forms = [f.strip() for f in args.forms.split(",") if f.strip()]
    launches = 0
    final_f64 = None
    rho_final = {}
    from nest_b200.exact_riemann import l1_rho_diagonal
    for form in forms:
        if ws > 1 or args.slab_path:
            r = run_slabs(args, ws, rank, form, cfl, st)
            launches += 2 * args.steps
            ab = alg_bytes_per_cell(form)
            m1, m2 = float(np.mean(r["k1"])), float(np.mean(r["k2"]))
            dom, dom_ms = ("stage2", m2) if m2 >= m1 else ("stage1", m1)
            cl = r["cells_local"]
            achieved = ab[dom] * cl / (dom_ms * 1e-3) / 1e9
            tr = traffic_from_profiles(form, n)
            value = ws * cl * 2 / (r["ms"] * 1e-3)
            results[form] = {
                "value": value, "ms_per_step": r["ms"], "sim_time": r["tsim"], "steps": r["steps"],
                "tiling": {"rows_per_tile": r["tiling"][0], "warps_per_block": r["tiling"][1]},
                "kernel_ms": {"stage1": m1, "stage2": m2},
                "hbm_gbs_step": value / ws * ab["per_cell_update"] / 1e9,
                "roofline": {"bound": "hbm", "kernel": kernel_name(form, dom), "achieved": achieved, "peak": hbm,
                             "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                             "alg_bytes_per_launch": ab[dom] * cl, "traffic": (tr or {}).get(dom)},
                "window": r["window"],
            }
            if "e2e" in r:
                results[form]["e2e"] = r["e2e"]
            continue
        prec, flags = form_args(form)
        U = U64.astype(np.float32) if prec == nb.F32 else U64
        s = nb.Solver(2, n, n, bc=nb.BC_OUTFLOW, precision=prec, flags=flags, stream=st.cuda_stream)
        tiling = tuple(int(v) for v in args.tiling.split(",")) if args.tiling else best_tiling(tune_form(form), n, n)
        s.set_tiling(*tiling)
        s.upload(U)
        s.step(args.warmup, cfl)
        s.sync()
        # timed region: K steps from the initial state, one event between kernels
        s.upload(U)
        s.reset_time()
        barrier(ws)
        torch.cuda.synchronize()
        t0 = time.time()
        k1, k2, total = s.step_profiled(args.steps, cfl)
        torch.cuda.synchronize()
        t1 = time.time()
        barrier(ws)
        launches += 2 * args.steps
        ms = allmax(ws, total) / args.steps
        tsim, nst = s.time()
        # the same K steps replayed through the captured CUDA graphs
        s.upload(U)
        s.reset_time()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        s.step(args.steps, cfl)
        e1.record(st)
        e1.synchronize()
        graph_ms = e0.elapsed_time(e1) / args.steps
        Ufin = s.download()
        rho_final[form] = Ufin[0, 2:-2, 2:-2].astype(np.float64)
        if form == "f64":
            final_f64 = (Ufin, tsim, nst)
        del Ufin
        ab = alg_bytes_per_cell(form)
        m1, m2 = float(np.mean(k1)), float(np.mean(k2))
        dom, dom_ms = ("stage2", m2) if m2 >= m1 else ("stage1", m1)
        achieved = ab[dom] * cells / (dom_ms * 1e-3) / 1e9
        tr = traffic_from_profiles(form, n)
        value = ws * cells * 2 * args.steps / (ms * args.steps * 1e-3)
        results[form] = {
            "value": value, "ms_per_step": ms, "graph_ms_per_step": graph_ms,
            "sim_time": tsim, "steps": nst, "tiling": {"rows_per_tile": tiling[0], "warps_per_block": tiling[1]},
            "kernel_ms": {"stage1": m1, "stage2": m2},
            "hbm_gbs_step": value / ws * ab["per_cell_update"] / 1e9,
            "roofline": {"bound": "hbm", "kernel": kernel_name(form, dom), "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": ab[dom] * cells,
                         "traffic": (tr or {}).get(dom)},
            "window": (t0, t1),
            "l1_rho_vs_exact": l1_rho_diagonal(rho_final[form], tsim, margin=0.05),
        }
        if not args.no_e2e:
            results[form]["e2e"] = e2e_run(s, U, args.steps, cfl, st, cells, ws)
        s.close()
        del s
    clocks.stop()
    for f in ("f32", "f32plain"):
        if f in rho_final and "f64" in rho_final:
            d = np.abs(rho_final[f] - rho_final["f64"])
            results[f]["rho_vs_f64"] = {"max_abs": float(d.max()), "l1": float(d.mean())}
    rho_final.clear()
    head = forms[0]
    r = results[head]
    clk = clocks.summary(min(x["window"][0] for x in results.values()), max(x["window"][1] for x in results.values()))
    for x in results.values():
        x.pop("window")
    out = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if head.startswith("f32") else "f64", "data": "synthetic",
        "config": workload_config(n, ws, head, args.slab_path),
        "roofline": r["roofline"],
        "forms": results,
        "e2e": r.get("e2e"),
        "clocks": clk,
        "gpu_launches": launches,
    }
    if not args.no_extras:
        ex = {e.strip() for e in args.extras.split(",")}
        if "batched" in ex:
            out["batched_kh"] = bench_batch(args, ws)
        if "adjoint1d" in ex:
            out["adjoint_1d"] = bench_adjoint(args)
        if "sod1d" in ex:
            out["sod_1d"] = bench_sod1d()
        if "adjoint2d" in ex and not args.no_adjoint2d:
            out["adjoint_2d_kh"] = bench_adjoint2d(args)
        if "adjoint2d_study" in ex:
            out["adjoint_2d_study"] = bench_adjoint2d_study(args)
        out["gpu_launches_extras"] = sum(out[k]["launches"] for k in ("batched_kh", "adjoint_1d", "sod_1d")
                                         if k in out)
    if ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"], parity = cpu_baseline(n, args.cpu_seconds, args.steps, final_f64)
        if parity is not None:
            results["f64"]["parity_vs_oracle"] = parity
            results["f64"]["max_rel_diff_vs_oracle"] = parity["max_rel_diff"]
    return out


def bench_batch(args, ws):
    """Batched Kelvin-Helmholtz: `count` independent periodic problems with
    sides drawn uniformly from {64, ..., 1024} (seed 0), FP32 state with FP64
    totals and repair, one persistent launch per stage, steps replayed from
    captured CUDA graphs; K = batch_steps steps per problem."""
    import torch
    import nest_b200 as nb
    from nest_b200.problems import kelvin_helmholtz, kh_sizes
    nx, ny = kh_sizes(args.batch_count, seed=0)
    rank = int(os.environ.get("RANK", "0"))
    ids = np.arange(rank, len(nx), ws)          # problems are independent: rank r takes r, r+ws, ...
    nx, ny = nx[ids], ny[ids]
    st = torch.cuda.Stream()
    from nest_b200.tuning import best_batch_tiling
    b = nb.Batch(nx, ny, precision=nb.F32, flags=nb.FLAG_TOTALS | nb.FLAG_REPAIR, stream=st.cuda_stream)
    ics = [kelvin_helmholtz(int(nx[p]), int(ny[p]), seed=1 + int(ids[p])).astype(np.float32) for p in range(len(nx))]
    for p, U in enumerate(ics):
        b.upload(p, U)
    tiling = best_batch_tiling(b, nx, ny)  # may advance the states: re-upload below
    b.set_tiling(*tiling)
    for p, U in enumerate(ics):
        b.upload(p, U)
    b.reset()
    del ics
    cells, items, blocks = b.info()
    b.step(2, 0.4)
    torch.cuda.synchronize()
    t0 = b.totals().copy()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    b.step(args.batch_steps, 0.4)
    e1.record(st)
    e1.synchronize()
    ms = allmax(ws, e0.elapsed_time(e1))
    cells = allsum(ws, cells)
    times, steps = b.times()
    tot = b.totals()
    drift = np.abs(tot - t0).max(axis=0) / np.maximum(np.abs(t0).max(axis=0), 1e-300)
    value = cells * 2 * args.batch_steps / (ms * 1e-3)
    # accuracy: the same problems advanced the same 2 + K steps by the plain
    # FP64 form (one FP64 batch); L1(rho) of every problem against it
    acc = batch_vs_f64(b, nx, ny, ids, 2 + args.batch_steps, times, st)
    b.close()
    return {"value": value, "unit": UNIT, "problems": args.batch_count, "problems_per_rank": int(len(nx)),
            "l1_rho_vs_f64": acc,
            "sharding": f"by problem over {ws} rank(s), no collective", "cells": int(cells), "steps": args.batch_steps,
            "ms_total": ms, "ms_per_step": ms / args.batch_steps, "work_items": items, "persistent_blocks": blocks,
            "hbm_gbs_equiv_per_gpu": value / ws * 40 / 1e9, "sim_time_range": [float(times.min()), float(times.max())],
            "fp64_totals_rel_drift": {"mass": float(drift[0]), "energy": float(drift[3])},
            "tiling": {"rows_per_item": tiling[0], "warps_per_block": tiling[1], "blocks_per_sm": tiling[2]},
            "launches": 4 * args.batch_steps, "dtype": "f32 (FP64 totals, time, repair)"}


def batch_vs_f64(b32, nx, ny, ids, nsteps, times32, st):
    """L1(rho) of each problem of an FP32 batch against the plain FP64 form
    run from the same initial states for the same number of steps (untimed)."""
    import nest_b200 as nb
    from nest_b200.problems import kelvin_helmholtz
    b64 = nb.Batch(nx, ny, precision=nb.F64, stream=st.cuda_stream)
    for p in range(len(nx)):
        b64.upload(p, kelvin_helmholtz(int(nx[p]), int(ny[p]), seed=1 + int(ids[p])))
    b64.step(nsteps, 0.4)
    t64, _ = b64.times()
    l1, rel = [], []
    for p in range(len(nx)):
        r64 = b64.download(p, nb.LAYOUT_INTERIOR)[0]
        r32 = b32.download(p, nb.LAYOUT_INTERIOR)[0].astype(np.float64)
        d = float(np.mean(np.abs(r32 - r64)))
        l1.append(d)
        rel.append(d / float(np.mean(np.abs(r64))))
    b64.close()
    l1, rel = np.array(l1), np.array(rel)
    return {"steps": nsteps, "max": float(l1.max()), "median": float(np.median(l1)),
            "max_relative_to_mean_rho": float(rel.max()),
            "sim_time_rel_diff_max": float(np.max(np.abs(times32 - t64) / t64)),
            "reference": "plain FP64 form, same initial states and step count"}


def bench_adjoint(args):
    """1D adjoint workload: N periodic cells, Fourier initial state (seeds 1
    and 2), K steps at CFL 0.4, loss 1/2 sum (rho_T - rho_target)^2 dx,
    checkpoint every 64 steps; forward sweep (CFL, dts recorded) and
    backward sweep (segment recompute + adjoint) timed separately."""
    import nest_b200 as nb
    from nest_b200.adjoint import Adjoint
    from nest_b200.problems import fourier_fields_1d, prim_to_cons_1d
    n, K = args.adjoint_n, args.adjoint_steps
    U0 = prim_to_cons_1d(*fourier_fields_1d(n, seed=1))
    tgt = prim_to_cons_1d(*fourier_fields_1d(n, seed=2))[0, 2:-2]
    s = nb.Solver(1, n, bc=nb.BC_PERIODIC, flags=nb.FLAG_NO_RESIDENT)
    s.upload(U0)
    a = Adjoint(s, K, 0, 64)
    a.forward(0.4)  # warm (graph capture, first launches)
    s.upload(U0)
    a = Adjoint(s, K, 0, 64)
    a.forward(0.4)
    UT = s.download()
    lam = np.zeros_like(UT)
    lam[0, 2:-2] = (UT[0, 2:-2] - tgt) / n
    lam0 = a.backward(lam)
    st = a.stats()
    fwd, bwd = st["forward_ms"], st["backward_ms"]
    fd = fd_check_1d(lambda: nb.Solver(1, n, bc=nb.BC_PERIODIC, flags=nb.FLAG_NO_RESIDENT), U0, tgt, n, K,
                     a.dts(), lam0, ndir=args.fd_directions) if args.fd_directions > 0 else None
    # the FP32 form: FP32 forward and reverse stages on the FP64 run's loss;
    # its gradient against the FP64 adjoint gradient
    s32 = nb.Solver(1, n, bc=nb.BC_PERIODIC, precision=nb.F32)
    s32.upload(U0.astype(np.float32))
    a32 = Adjoint(s32, K, 0, 64)
    a32.forward(0.4)  # warm
    s32.upload(U0.astype(np.float32))
    a32 = Adjoint(s32, K, 0, 64)
    a32.forward(0.4)
    UT32 = s32.download().astype(np.float64)
    lam32 = np.zeros_like(UT32)
    lam32[0, 2:-2] = (UT32[0, 2:-2] - tgt) / n
    g32 = a32.backward(lam32.astype(np.float32)).astype(np.float64)[:, 2:-2]
    st32 = a32.stats()
    g64 = lam0[:, 2:-2]
    f32 = {"forward_ms": st32["forward_ms"], "backward_ms": st32["backward_ms"],
           "adjoint_over_forward": st32["backward_ms"] / st32["forward_ms"],
           "grad_rel_l2_vs_f64": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
           "grad_cosine_vs_f64": float(np.sum(g32 * g64) / (np.linalg.norm(g32) * np.linalg.norm(g64)))}
    a32.close()
    s32.close()
    return {"n": n, "steps": K, "checkpoint_every": 64, "forward_ms": fwd, "backward_ms": bwd, "fd_check": fd,
            "adjoint_over_forward": bwd / fwd, "gradient_over_forward": (fwd + bwd) / fwd,
            "recomputed_steps": st["recomputed_steps"], "checkpoint_mb": st["checkpoint_bytes"] / 1e6,
            "launches": 2 * (K + 2 * K), "dtype": "f64", "f32": f32}


def bench_sod1d(reps: int = 20):
    """1D Sod: N = 1024, outflow, CFL 0.4 to t = 0.2, FP64 (one thread-block
    cluster runs the whole loop).  Device time of run_to from the initial state;
    L1(rho) against the exact solution."""
    import torch
    import nest_b200 as nb
    from nest_b200.exact_riemann import l1_rho_1d
    from nest_b200.problems import sod_1d
    n = 1024
    s = nb.Solver(1, n, bc=nb.BC_OUTFLOW)
    U0 = sod_1d(n)
    ext = torch.cuda.ExternalStream(s.stream_ptr())
    s.upload(U0)
    s.run_to(0.2, 0.4)
    ms = []
    for _ in range(reps):
        s.upload(U0)
        s.reset_time()
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        steps = s.run_to(0.2, 0.4)
        e1.record(ext)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    t, _ = s.time()
    rho = s.download()[0, 2:-2]
    m = float(np.median(ms))
    s.close()
    return {"n": n, "bc": "outflow", "cfl": 0.4, "t_final": t, "steps": steps, "ms": m,
            "value": n * steps * 2 / (m * 1e-3), "unit": UNIT, "l1_rho_vs_exact": l1_rho_1d(rho, t),
            "launches": 1, "dtype": "f64",
            "kernel": "k1d_cluster (one thread-block cluster of 16 CTAs runs the whole loop in shared memory)"}


def ke_v(U, nx, ny):
    """L = integral of 1/2 rho v^2 dA over the interior and dL/dU (extended layout)."""
    r, mv = U[0, 2:-2, 2:-2].astype(np.float64), U[2, 2:-2, 2:-2].astype(np.float64)
    v = mv / r
    dA = 1.0 / (nx * ny)
    lam = np.zeros(U.shape)
    lam[0, 2:-2, 2:-2] = -0.5 * v * v * dA
    lam[2, 2:-2, 2:-2] = v * dA
    return 0.5 * float(np.sum(r * v * v)) * dA, lam


def bench_adjoint2d(args):
    """Kelvin-Helmholtz on one periodic n x n grid (seed 1), K steps at CFL
    0.4, loss = integral of 1/2 rho v^2 dA at the end, binomial
    checkpointing with as many snapshots as fit in 40 GB; gradient with
    respect to the initial v field (rho, u, p held), FP64 and FP32; the FP32
    gradient is compared with the FP64 one."""
    import nest_b200 as nb
    from nest_b200.adjoint import BINOMIAL, Adjoint
    from nest_b200.problems import kelvin_helmholtz
    n, K = args.adjoint2d_n, args.adjoint2d_steps
    forms = getattr(args, "adjoint2d_forms", "f64,f32").split(",")
    U0 = kelvin_helmholtz(n, n, seed=1)
    out, grads = {}, {}
    for form, prec, dt in (("f64", nb.F64, np.float64), ("f32", nb.F32, np.float32)):
        if form not in forms:
            continue
        s = nb.Solver(2, n, n, bc=nb.BC_PERIODIC, precision=prec)
        _, pitch, vs = s.state_ptr()
        slots = int(min(K, 40e9 // (4 * vs * np.dtype(dt).itemsize)))
        s.upload(U0.astype(dt))
        a = Adjoint(s, K, BINOMIAL, slots)
        a.forward(0.4)
        UT = s.download()
        L, lam = ke_v(UT, n, n)
        lam0 = a.backward(lam.astype(dt)).astype(np.float64)
        st = a.stats()
        r0, ru0, rv0 = U0[0, 2:-2, 2:-2], U0[1, 2:-2, 2:-2], U0[2, 2:-2, 2:-2]
        # dL/dv0 with rho, u, p held: d(rho v)/dv = rho, dE/dv = rho v
        grads[form] = lam0[2, 2:-2, 2:-2] * r0 + lam0[3, 2:-2, 2:-2] * rv0
        out[form] = {"forward_ms": st["forward_ms"], "backward_ms": st["backward_ms"],
                     "adjoint_over_forward": st["backward_ms"] / st["forward_ms"],
                     "recomputed_steps": st["recomputed_steps"], "snapshots": slots,
                     "checkpoint_gb": st["checkpoint_bytes"] / 1e9, "loss": L}
        a.close()
        s.close()
    if len(grads) == 2:
        g64, g32 = grads["f64"], grads["f32"]
        out["f32_vs_f64_grad_rel_l2"] = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
        out["f32_vs_f64_grad_cosine"] = float(np.sum(g32 * g64) / (np.linalg.norm(g32) * np.linalg.norm(g64)))
    out["grad_l2"] = {k: float(np.linalg.norm(v)) for k, v in grads.items()}
    out.update({"n": n, "steps": K, "policy": "binomial (snapshots fitting 40 GB)",
                "loss": "integral of 1/2 rho v^2 dA at t_end", "gradient": "d loss / d v(t=0)",
                "launches": None})
    return out


def kh_grad_v(U0, n, K, prec_np, slots_budget=40e9):
    """d loss / d v(t=0) of the config-5 loss (integral of 1/2 rho v^2 dA at
    step K) through the checkpointed adjoint; returns (gradient, dts, stats
    with the loss and the final density)."""
    import nest_b200 as nb
    from nest_b200.adjoint import BINOMIAL, Adjoint
    prec = nb.F64 if prec_np == np.float64 else nb.F32
    s = nb.Solver(2, n, n, bc=nb.BC_PERIODIC, precision=prec)
    _, pitch, vs = s.state_ptr()
    slots = int(min(K, slots_budget // (4 * vs * np.dtype(prec_np).itemsize)))
    s.upload(U0.astype(prec_np))
    a = Adjoint(s, K, BINOMIAL, slots)
    a.forward(0.4)
    UT = s.download()
    L, lam = ke_v(UT, n, n)
    lam0 = a.backward(lam.astype(prec_np)).astype(np.float64)
    g = lam0[2, 2:-2, 2:-2] * U0[0, 2:-2, 2:-2] + lam0[3, 2:-2, 2:-2] * U0[2, 2:-2, 2:-2]
    dts, st = a.dts(), a.stats()
    a.close()
    s.close()
    return g, dts, dict(st, loss=L, rho=UT[0, 2:-2, 2:-2].astype(np.float64))


def bench_adjoint2d_study(args):
    """Config-5 gradient study (Kelvin-Helmholtz, n x n periodic, seed 1).
    For each horizon K: the FP32 gradient against the FP64 gradient, and, as
    controls, FP64 gradients of perturbed initial states against the FP64
    gradient: the state rounded once through FP32 (about 1e-8 relative) and
    seeded relative noise of 1e-6 and 1e-5 on every conserved field.  Each
    run also reports how far its final density lies from the FP64 run's
    (relative L2), so the FP32 trajectory's deviation can be set beside the
    controls'.  If a control whose trajectory deviates as much as FP32's
    decorrelates like FP32 does, the disagreement is the flow's sensitivity,
    not an error of either adjoint.  At the longest horizon the FP64 gradient
    is also checked by central differences along smooth directions of the
    initial v field (dts frozen from the FP64 forward sweep)."""
    import nest_b200 as nb
    from nest_b200.problems import kelvin_helmholtz
    n = args.adjoint2d_n
    hs = [int(x) for x in args.adjoint2d_horizons.split(",")]
    U0 = kelvin_helmholtz(n, n, seed=1)
    rng = np.random.default_rng(11)
    noise = rng.standard_normal(U0.shape)
    controls = {"f64_rounded_ic": U0.astype(np.float32).astype(np.float64),
                "f64_noise_1e-6": U0 * (1 + 1e-6 * noise), "f64_noise_1e-5": U0 * (1 + 1e-5 * noise)}

    def cmp(a, b):
        return {"rel_l2": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
                "cosine": float(np.sum(a * b) / (np.linalg.norm(a) * np.linalg.norm(b)))}

    out = {"n": n, "horizons": {}}
    last = None
    for K in hs:
        g64, dts, st64 = kh_grad_v(U0, n, K, np.float64)
        runs = {"f32": kh_grad_v(U0, n, K, np.float32)}
        for name, Uc in controls.items():
            runs[name] = kh_grad_v(Uc, n, K, np.float64)
        h = {"grad_l2": {"f64": float(np.linalg.norm(g64))}}
        for name, (g, _, st) in runs.items():
            h[name + "_vs_f64"] = dict(cmp(g, g64), final_rho_rel_l2=float(
                np.linalg.norm(st["rho"] - st64["rho"]) / np.linalg.norm(st64["rho"])))
            h["grad_l2"][name] = float(np.linalg.norm(g))
        out["horizons"][str(K)] = h
        last = (K, g64, dts, st64["loss"])
    K, g64, dts, L0 = last
    x = (np.arange(n) + 0.5) / n
    fd = []
    for (m, k, ph) in ((1, 2, 0.1), (2, 1, 0.35), (3, 3, 0.7)):
        d = np.outer(np.sin(2 * np.pi * (m * x + ph)), np.cos(2 * np.pi * k * x))
        ad = float(np.sum(g64 * d))

        def L(eps):
            U = U0[:, 2:-2, 2:-2].copy()
            r, mv = U[0], U[2]
            U[3] = U[3] + mv * eps * d + 0.5 * r * (eps * d) ** 2
            U[2] = mv + r * eps * d
            s = nb.Solver(2, n, n, bc=nb.BC_PERIODIC, precision=nb.F64)
            s.freeze_dts(dts)
            s.upload(U, nb.LAYOUT_INTERIOR)
            s.step(K, 0.4)
            val = ke_v(s.download(), n, n)[0]
            s.close()
            return val
        row = {"mode": [m, k], "adjoint": ad}
        for eps in (1e-4, 1e-6):
            f = (L(eps) - L(-eps)) / (2 * eps)
            row[f"fd_eps_{eps:g}"] = f
            row[f"rel_err_eps_{eps:g}"] = abs(ad - f) / max(abs(f), 1e-300)
        fd.append(row)
    out["fd_check_f64"] = {"steps": K, "directions": fd}
    return out


def fd_check_1d(s_factory, U0, tgt, n, K, dts, lam0, ndir: int = 32, eps: float = 1e-8):
    """Directional derivatives of the 1D loss by central differences (dts
    frozen) on `ndir` smooth random directions against the adjoint's."""
    rng = np.random.default_rng(5)
    x = (np.arange(n) + 0.5) / n
    rel = []
    for _ in range(ndir):
        d = np.zeros_like(U0)
        for k in range(3):
            c = rng.standard_normal(4)
            d[k, 2:-2] = sum(c[m] * np.sin(2 * np.pi * (m + 1) * x + c[(m + 1) % 4]) for m in range(4))
        vals = []
        for sgn in (1.0, -1.0):
            s = s_factory()
            s.freeze_dts(dts)
            s.upload(U0 + sgn * eps * d)
            s.step(K, 0.4)
            r = s.download()[0, 2:-2] - tgt
            vals.append(0.5 * float(np.sum(r * r)) / n)
            s.close()
        fd = (vals[0] - vals[1]) / (2 * eps)
        ad = float(np.sum(lam0[:, 2:-2] * d[:, 2:-2]))
        rel.append(abs(ad - fd) / max(abs(fd), 1e-300))
    return {"directions": ndir, "eps": eps, "rel_err_median": float(np.median(rel)), "rel_err_max": float(np.max(rel))}


def e2e_run(s, U, steps, cfl, st, cells, ws):
    """Through the public API with pinned host buffers: upload the initial
    state, run the K steps, download the final state and read the clock."""
    import torch
    import nest_b200 as nb
    tdt = torch.float32 if U.dtype == np.float32 else torch.float64
    hin = torch.empty(U.shape, dtype=tdt, pin_memory=True)
    hin.numpy()[...] = U
    hout = torch.empty(U.shape, dtype=tdt, pin_memory=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    nb.solver.check(nb._capi.lib.nest_solver_upload(s._h, hin.data_ptr(), nb.LAYOUT_EXTENDED), "upload")
    s.reset_time()
    s.step(steps, cfl)
    nb.solver.check(nb._capi.lib.nest_solver_download(s._h, hout.data_ptr(), nb.LAYOUT_EXTENDED), "download")
    t, k = s.time()
    e1.record(st)
    e1.synchronize()
    ms = allmax(ws, e0.elapsed_time(e1))
    nbytes = U.nbytes
    return {"value": ws * cells * 2 * steps / (ms * 1e-3), "unit": UNIT, "ms_total": ms,
            "h2d_bytes_per_step": nbytes / steps, "d2h_bytes_per_step": (nbytes + 32) / steps,
            "api": "nest_solver_upload -> nest_solver_step -> nest_solver_download -> nest_solver_time"}


# ---------------------------------------------------------------------------
# CPU side (oracle port of the same scheme on the host cores)
# ---------------------------------------------------------------------------

def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(n: int, budget_s: float, steps: int, final_f64=None):
    """FP64 scheme on the host cores (the oracle, OpenMP on every host core)
    from the workload's initial state: after one untimed step, S steps sized
    to about budget_s seconds are timed (the baseline); when the bench timed
    the FP64 form, the oracle then runs on to the bench's K steps and its
    state is compared with the GPU's final state cell for cell (the FP64
    form's parity check at the full size, all four variables, ghost cells
    excluded).  Returns (cpu_baseline, parity or None)."""
    from oracle.oracle import BC_OUTFLOW, Oracle
    from nest_b200.problems import riemann_2d
    orc = Oracle()
    th = host_threads()
    orc.set_threads(th)
    U = np.ascontiguousarray(riemann_2d(n, n))
    run = lambda k: orc.run2d(U, n, n, 2, 1 / n, 1 / n, 1.4, 0.4, nsteps=k, bc=BC_OUTFLOW, record_dts=True)
    dts = []
    t0 = time.perf_counter()
    dts += list(run(1)[2])
    t1 = time.perf_counter() - t0
    S = int(max(1, min(50, budget_s / max(t1, 1e-6) - 1)))
    if final_f64 is not None:
        S = max(1, min(S, steps - 1))
    t0 = time.perf_counter()
    dts += list(run(S)[2])
    el = time.perf_counter() - t0
    base = {"value": n * n * 2 * S / el, "unit": UNIT, "cores": th, "kind": "port",
            "sample": f"{S} RK2 steps (after 1 untimed) of the {n}x{n} FP64 diagonal Riemann problem, "
                      f"oracle/euler_oracle.c with OpenMP ({th} threads), {el:.1f} s"}
    if final_f64 is None:
        return base, None
    Ug, tg, kg = final_f64
    rest = steps - 1 - S
    if rest > 0:
        dts += list(run(rest)[2])
    tc = 0.0
    for d in dts:  # the solver's clock: time += dt each step
        tc += d
    a, b = Ug[:, 2:-2, 2:-2], U[:, 2:-2, 2:-2]
    diff = np.abs(a - b)
    rel = diff / np.maximum(np.abs(b), 1e-300)
    parity = {"steps": len(dts), "gpu_steps": int(kg), "bit_exact": bool(np.array_equal(a, b)),
              "max_rel_diff": float(rel.max()), "max_abs_diff": float(diff.max()),
              "time_gpu": float(tg), "time_oracle": tc, "time_equal": bool(tg == tc),
              "oracle": f"oracle/euler_oracle.c, {th} threads, {len(dts)} steps from the initial state"}
    return base, parity


def run_reference(args, rank):
    """CPU arm: each step is one RK2 step of a sample of the workload the CUDA
    arm runs at this world size -- the first nx_s rows of the (N n) x n grid
    (N = world size) as an outflow domain -- sized from a one-step probe so
    the whole run stays within minutes."""
    from oracle.oracle import BC_OUTFLOW, Oracle
    riemann_2d = load_problems().riemann_2d
    orc = Oracle()
    th = host_threads()
    orc.set_threads(th)
    ws = max(1, int(os.environ.get("WORLD_SIZE", args.gpus)))
    n = args.n
    nxg = ws * n
    dx, dy = 1 / nxg, 1 / n
    nx_s = min(nxg, n)
    U = np.ascontiguousarray(riemann_2d(nxg, n, rows=(0, nx_s)))
    t0 = time.perf_counter()
    orc.run2d(U, nx_s, n, 2, dx, dy, 1.4, 0.4, nsteps=1, bc=BC_OUTFLOW)
    t1 = time.perf_counter() - t0
    per_step_budget = 90.0 / max(1, args.steps + args.warmup)
    if t1 > per_step_budget:
        nx_s = max(64, int(nx_s * per_step_budget / t1) // 64 * 64)
    Us = np.ascontiguousarray(riemann_2d(nxg, n, rows=(0, nx_s)))
    orc.run2d(Us, nx_s, n, 2, dx, dy, 1.4, 0.4, nsteps=max(1, args.warmup), bc=BC_OUTFLOW)
    Us = np.ascontiguousarray(riemann_2d(nxg, n, rows=(0, nx_s)))
    t0 = time.perf_counter()
    orc.run2d(Us, nx_s, n, 2, dx, dy, 1.4, 0.4, nsteps=args.steps, bc=BC_OUTFLOW)
    el = time.perf_counter() - t0
    value = nx_s * n * 2 * args.steps / el
    sample = (f"{args.steps} RK2 steps of a {nx_s}x{n} slab of the {nxg}x{n} FP64 diagonal Riemann problem, "
              f"oracle/euler_oracle.c (the scheme's CPU restatement; nest has no 2D RK2), OpenMP {th} threads")
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(n, ws, "f64", False),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": th, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args, rank)), flush=True)
        return 0
    ws, rank, local = dist_setup(args.slab_path)
    if ws > 1 or args.slab_path:
        import torch
        torch.cuda.set_device(local)
    out = run_ours(args, ws, rank, local)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if ws > 1 or args.slab_path:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
