"""Build recipe of the CUDA library (libnest_b200.so) for sm_100a.

Each translation unit gets its own floating-point flags:
  euler1d.cu, euler2d_f64.cu  -fmad=false  (FP64 plain form: bit-exact with
                                            nest's CPU operation order)
  euler1d_f32.cu, euler2d_f32*.cu
                              -use_fast_math (FP32 form)
  capi.cpp                    host runtime and C ABI (compiled as CUDA C++)
The library is built in-tree (nest_b200/lib/) so that it travels with the
repository snapshot; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libnest_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC", "-I", str(PKG.parent / "include")]

UNITS = {
    "euler1d.cu": ["-fmad=false"],
    "euler1d_f32.cu": ["-use_fast_math"],
    "euler2d_f64.cu": ["-fmad=false"],
    "euler2d_f64r.cu": ["-fmad=false"],
    "euler2d_f32.cu": ["-use_fast_math"],
    "euler2d_f32x2.cu": ["-use_fast_math"],
    "euler2d_compat.cu": ["-fmad=false"],
    "capi.cpp": ["-x", "cu"],
    "noalloc.cu": [],
    "adjoint1d.cu": [],
    "adjoint1d_f32.cu": ["-use_fast_math"],
    "adjoint.cpp": ["-x", "cu"],
    "exchange.cu": [],
    "adjoint2d.cu": [],
    "adjoint2d_f32.cu": ["-use_fast_math"],
    "adjoint2d_f32x2.cu": ["-use_fast_math"],
    "adjoint2d_f64rm.cu": ["-fmad=false"],
    "datio.cpp": ["-x", "cu", "-Xcompiler", "-ffp-contract=off"],
    "pipeline.cu": ["-fmad=false"],
    "slab.cpp": ["-x", "cu"],
}


def _headers():
    return list(SRC.glob("*.cuh")) + list(SRC.glob("*.h")) + [PKG.parent / "include" / "nest_b200.h"]


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _compile(unit: str, flags, verbose: bool) -> Path:
    obj = BUILD / (unit.replace(".", "_") + ".o")
    deps = [SRC / unit] + _headers() + [Path(__file__)]
    if not _stale(obj, deps):
        return obj
    cmd = [NVCC] + COMMON + flags + ["-c", str(SRC / unit), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr)
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), UNITS.items()))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
