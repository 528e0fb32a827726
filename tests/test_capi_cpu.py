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
    ]
    for kw in bad:
        with pytest.raises(nb.NestError) as e:
            nb.Solver(**kw)
        assert e.value.status in (1, 6)
    assert A.lib.nest_solver_step(None, 1, 0.4) == 1
    assert "null" in A.last_error()
    assert A.lib.nest_version() >= 10000
