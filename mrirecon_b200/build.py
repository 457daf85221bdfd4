"""Build the in-tree CUDA library ``libmrirecon_b200.so`` for sm_100a.

    python -m mrirecon_b200.build [--force] [--verbose]

Compiles every ``csrc/*.cu`` with nvcc (``-gencode arch=compute_100a,code=sm_100a``)
into objects under ``mrirecon_b200/_build`` and links them with cuFFT into
``mrirecon_b200/libmrirecon_b200.so``.  Rebuilds only what changed.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmrirecon_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


# Files whose kernels also run in grouped form (csrc/group.cuh): the compiler
# fuses no multiply into an add on its own there (every fused multiply-add is
# written as fmaf / fma), so a kernel and its grouped form, two compilations of
# the same source, round every operation alike and produce the same bits.
NO_FMAD = {"ncg.cu", "fft.cu"}


def _flags(src: str = ""):
    fmad = "-fmad=false" if os.path.basename(src) in NO_FMAD else "-fmad=true"
    return ["-O3", "-lineinfo", "-std=c++17", fmad, "-Xcompiler", "-fPIC",
            "-Xcompiler", "-O3", "--expt-relaxed-constexpr", "-I", os.path.join(PKG, "..", "include")] + ARCH


def _deps_mtime(src: str) -> float:
    hdrs = (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(PKG, "..", "include", "*.h")) +
            [os.path.abspath(__file__)])
    return max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in hdrs])


def _compile(src: str, force: bool, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime(src):
        return obj
    cmd = [nvcc()] + _flags(src) + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcufft"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
