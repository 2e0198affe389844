"""Builds the CUDA search core in-tree: rmblast_b200/lib/librmb_b200.so (sm_100a).

    python -m rmblast_b200.build        # or: from rmblast_b200.build import build; build()

nvcc cross-compiles for sm_100a without a GPU; the .so is written next to the package so it
travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "librmb_b200.so"
SOURCES = ["rmb_kernels.cu", "rmb_capi.cu", "rmb_glue.cpp", "rmb_io.cpp", "rmb_probe.cu", "rmb_sched.cu"]
HEADERS = ["rmb_device.cuh", "rmb_dust.cuh", "rmb_prelim_stream.cuh", "rmb_sched.cuh", "rmb_ungapped.cuh", "rmb_kernels.hpp", "rmb_glue.hpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [PKG.parent / "include" / "rmb_gpu.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    objs, procs = [], []
    for s in SOURCES:  # the sources compile concurrently
        o = LIB_DIR / (Path(s).stem + ".o")
        cmd = [nvcc(), *GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
               "-I", str(PKG.parent / "include"), "-c", str(CSRC / s), "-o", str(o)]
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(str(o))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [nvcc(), *GENCODE, "-shared", "-o", str(LIB), *objs, "-lcudart", "-Xcompiler", "-pthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
