"""The C-ABI library loads and exports what include/*.h declares; argument
validation works without a GPU (no compute calls here)."""
from __future__ import annotations

import ctypes as C
import re

import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\([^;]*\)\s*;", text, flags=re.M):
            if m.group(1) not in ("if", "while", "for", "sizeof"):
                names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_nest_abi():
    names = declared_functions()
    for n in ["euler1d_gpu_create", "euler1d_gpu_destroy", "euler1d_gpu_upload", "euler1d_gpu_download",
              "euler1d_gpu_compute_dt", "euler1d_gpu_rk2_step", "euler1d_gpu_run", "euler1d_gpu_run_timed"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    import nest_b200
    lib = C.CDLL(str(nest_b200.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_invalid_arguments_rejected_without_gpu():
    import nest_b200 as nb
    from nest_b200 import _capi as A
    bad = [
        dict(dim=3, nx=8, ny=8),
        dict(dim=2, nx=2, ny=8),
        dict(dim=2, nx=8, ny=8, gamma=1.0),
        dict(dim=1, nx=16, halo=1),
        dict(dim=2, nx=8, ny=8, halo=3),
        dict(dim=1, nx=16, precision=A.F32, flags=A.FLAG_TOTALS),
        dict(dim=2, nx=8, ny=8, dx=-1.0),
        dict(dim=2, nx=8, ny=8, dy=float("nan")),
        dict(dim=2, nx=65536, ny=32769),                       # more than 2^31 cells
        dict(dim=2, nx=8, ny=8, precision=7),
        dict(dim=2, nx=8, ny=8, bc=(A.BC_OUTFLOW, 5)),
        dict(dim=1, nx=16, bc=(5, 5)),
        dict(dim=1, nx=16, flags=A.FLAG_SPLIT_COMPAT),         # nest's split sweeps are 2D FP64
        dict(dim=2, nx=8, ny=8, precision=A.F32, flags=A.FLAG_SPLIT_COMPAT),
        dict(dim=2, nx=8, ny=8, flags=A.FLAG_SPLIT_COMPAT | A.FLAG_TOTALS),
        dict(dim=2, nx=8, ny=8, flags=A.FLAG_LIMITER_MC | A.FLAG_LIMITER_NONE),
    ]
    for kw in bad:
        with pytest.raises(nb.NestError) as e:
            nb.Solver(**kw)
        assert e.value.status in (1, 6)
    assert A.lib.nest_solver_step(None, 1, 0.4) == 1
    assert "null" in A.last_error()
    assert A.lib.nest_version() >= 10000


def test_dropin_abi_refuses_bad_input_without_gpu():
    """nest's euler1d_gpu_* entry points bound the way a nest maintainer would
    bind them (a ctypes stub of its own, not the package's wrapper): bad sizes,
    spacing, gamma or halo give NULL and a message instead of nest's C++
    exception through extern "C" (src/backend_cuda/euler1d_solver.cu:24-29),
    and every call on a null handle is refused without touching the device."""
    import nest_b200
    lib = C.CDLL(str(nest_b200.LIB_PATH))
    vp, dp = C.c_void_p, C.POINTER(C.c_double)
    lib.euler1d_gpu_create.restype, lib.euler1d_gpu_create.argtypes = vp, [C.c_int, C.c_int, C.c_double, C.c_double]
    lib.euler1d_gpu_destroy.restype, lib.euler1d_gpu_destroy.argtypes = None, [vp]
    lib.euler1d_gpu_upload.restype, lib.euler1d_gpu_upload.argtypes = None, [vp, dp]
    lib.euler1d_gpu_download.restype, lib.euler1d_gpu_download.argtypes = None, [vp, dp]
    lib.euler1d_gpu_compute_dt.restype, lib.euler1d_gpu_compute_dt.argtypes = C.c_double, [vp, C.c_double]
    lib.euler1d_gpu_rk2_step.restype, lib.euler1d_gpu_rk2_step.argtypes = None, [vp, C.c_double]
    lib.euler1d_gpu_run.restype, lib.euler1d_gpu_run.argtypes = C.c_int, [vp, C.c_double, C.c_double]
    lib.euler1d_gpu_run_timed.restype = C.c_double
    lib.euler1d_gpu_run_timed.argtypes = [vp, C.c_double, C.c_double, C.POINTER(C.c_int)]
    lib.euler1d_gpu_status.restype, lib.euler1d_gpu_status.argtypes = C.c_int, [vp]
    lib.nest_last_error.restype = C.c_char_p
    invalid = 1  # NEST_ERR_INVALID
    for args, words in [((0, 2, 0.1, 1.4), "interior"), ((-8, 2, 0.1, 1.4), "interior"),
                        ((16, 1, 1 / 16, 1.4), "halo"), ((16, 2, 0.0, 1.4), "cell sizes"),
                        ((16, 2, float("nan"), 1.4), "cell sizes"), ((16, 2, 1 / 16, 1.0), "gamma")]:
        assert lib.euler1d_gpu_create(*args) is None, args
        assert words in lib.nest_last_error().decode(), (args, lib.nest_last_error())
    lib.euler1d_gpu_destroy(None)
    lib.euler1d_gpu_upload(None, None)
    lib.euler1d_gpu_download(None, None)
    lib.euler1d_gpu_rk2_step(None, 1e-3)
    assert lib.euler1d_gpu_compute_dt(None, 0.4) == 0.0
    assert lib.euler1d_gpu_run(None, 0.2, 0.4) == -1
    n = C.c_int(7)
    assert lib.euler1d_gpu_run_timed(None, 0.2, 0.4, C.byref(n)) == -1.0
    assert lib.euler1d_gpu_status(None) == invalid
    assert "null" in lib.nest_last_error().decode()


def test_other_constructors_reject_bad_input_without_gpu():
    """Batches, nest's patch exchange plans and device pipelines check their
    arguments on the host before any device call (so these run without a
    GPU): nest's exchange needs every patch to hold at least `halo` interior
    cells per axis (its halo copies read that far into the neighbour)."""
    import nest_b200 as nb
    from nest_b200 import _capi as A
    from nest_b200.batch import Batch
    from nest_b200.exchange import PeriodicExchange
    from nest_b200.pipeline import Pipeline
    for kw in [dict(nx=[], ny=[]), dict(nx=[64, 2], ny=[64, 64]), dict(nx=[64], ny=[64], gamma=1.0),
               dict(nx=[64], ny=[64], bc=(A.BC_PERIODIC, 5)), dict(nx=[64], ny=[64], precision=7)]:
        with pytest.raises(nb.NestError) as e:
            Batch(**kw)
        assert e.value.status == A.NEST_ERR_INVALID, kw
    with pytest.raises(nb.NestError) as e:
        Batch([64], [64], flags=A.FLAG_LIMITER_MC)
    assert e.value.status == A.NEST_ERR_UNSUPPORTED
    for kw in [dict(dim=3, nx=64, npx=2, nvars=3, halo=2), dict(dim=1, nx=64, npx=2, nvars=0, halo=2),
               dict(dim=1, nx=64, npx=2, nvars=3, halo=0), dict(dim=1, nx=3, npx=2, nvars=3, halo=2),
               dict(dim=2, nx=64, npx=2, nvars=4, halo=2, ny=64, npy=0),
               dict(dim=2, nx=64, npx=2, nvars=4, halo=2, ny=5, npy=3)]:
        with pytest.raises(nb.NestError) as e:
            PeriodicExchange(**kw)
        assert e.value.status == A.NEST_ERR_INVALID, kw
    for kw in [dict(dim=3, nx=64, npx=2), dict(dim=1, nx=64, npx=2, dx=-1.0), dict(dim=1, nx=64, npx=2, gamma=1.0),
               dict(dim=1, nx=64, npx=2, nwork=17), dict(dim=1, nx=64, npx=2, limiter=9),
               dict(dim=1, nx=3, npx=2)]:
        with pytest.raises(nb.NestError) as e:
            Pipeline(**kw)
        assert e.value.status == A.NEST_ERR_INVALID, kw
