"""Compile libcutcell_b200.so in-tree for sm_100a with nvcc.

Every kernel is built with --fmad=false (no a*b+c contraction) and IEEE division / square root,
so each expression rounds as the reference's CPU code does. Objects go to ``_build/``; the shared
library lands beside this file, where the package loads it from.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libcutcell_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-std=c++17",
                "-Xcompiler", "-fPIC"]
SOURCES = ["capi.cu", "mc.cu", "ms.cu", "plic.cu", "noalloc.cu", "learned.cu", "learned_api.cu", "batch.cu", "mesh.cu", "ms_mesh.cu", "plic_mesh.cu"]
HEADERS = ["cc_device.cuh", "cc_internal.h", "mc_cell.cuh", "ms_cell.cuh", "compact.cuh"]


def _inputs():
    files = [os.path.join(SRC, s) for s in SOURCES] + [os.path.join(SRC, h) for h in HEADERS]
    files.append(os.path.join(HERE, "..", "include", "cutcell_b200.h"))
    return files


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(f) > t for f in _inputs() if os.path.exists(f))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return OUT
    os.makedirs(BUILD, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        cmd = [NVCC] + FLAGS + ["-c", os.path.join(SRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = OUT + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
