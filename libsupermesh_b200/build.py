"""Builds the CUDA library libsupermesh_b200/lib/libsupermesh.so for sm_100a.

The library is one shared object holding every kernel and the C-ABI of
include/libsupermesh-c.h and include/libsupermesh-gpu.h.  It links the CUDA
runtime statically, so it loads without torch or any other package.  All
device code is compiled with -fmad=false: the FP64 geometry must not contract
multiplies and adds into FMAs, or clipped vertices would differ in the last
bit from the reference algorithm.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SRC = PKG / "csrc"
OUT = PKG / "lib" / "libsupermesh.so"
PROBE = PKG / "lib" / "liblsm_probe.so"
SOURCES = ["lsm_kernels.cu", "lsm_capi.cu", "lsm_noalloc.cu", "lsm_sched.cu"]
HEADERS = ["lsm_geom.cuh", "lsm_kernels.h", "lsm_sched.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [SRC / f for f in SOURCES + HEADERS] + list((ROOT / "include").glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-shared",
           "-Xcompiler", "-fPIC,-O2", "--cudart", "static", "-I", str(ROOT / "include"),
           *[str(SRC / f) for f in SOURCES], "-o", str(tmp)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


def build_probe(force: bool = False) -> Path:
    """Measurement probe used by bench.py (FP64 issue-rate ceiling, L2 flush)."""
    src = SRC / "lsm_probe.cu"
    if not force and PROBE.exists() and PROBE.stat().st_mtime >= src.stat().st_mtime:
        return PROBE
    PROBE.parent.mkdir(parents=True, exist_ok=True)
    tmp = PROBE.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "--cudart", "static",
                    str(src), "-o", str(tmp)], check=True)
    os.replace(tmp, PROBE)
    return PROBE


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    build_probe(force="--force" in sys.argv)
    print(OUT)
