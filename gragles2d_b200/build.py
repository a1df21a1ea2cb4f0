"""Builds ``libgg_b200.so`` (the C ABI of include/gg_step.h) for sm_100a.

The plain (FP64) kernels are compiled with ``--fmad=false`` so their sums and
products round exactly like the reference's host arithmetic; the batched
(FP32) kernels keep FMA contraction.  Host code is compiled without FMA
contraction as well (it builds the Gaussian multipliers and twiddles).

Usage: ``python -m gragles2d_b200.build [--force]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgg_b200.so")
OBJDIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", os.path.join(HERE, "..", "include")]
UNITS = {
    "gg_plain": ["--fmad=false"],
    "gg_batched": [],
    "gg_host": ["--fmad=false"],
    "gg_static": ["--fmad=false"],
}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources_mtime() -> float:
    mt = 0.0
    for root in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(root):
            mt = max(mt, os.path.getmtime(os.path.join(root, f)))
    return mt


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the extension in-tree if sources are newer; returns the .so path."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _sources_mtime():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()

    def compile_unit(name: str) -> str:
        obj = os.path.join(OBJDIR, name + ".o")
        cmd = [nvcc, *ARCH, *COMMON, *UNITS[name], "-c", os.path.join(CSRC, name + ".cu"), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(compile_unit, UNITS))
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", *objs, "-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
