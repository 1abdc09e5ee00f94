"""Build recipe of the native library ``multiflow3d_b200/libmf3d.so``.

Compiles the CUDA/C++ sources for sm_100a only, in-tree, with nvcc:
``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -fmad=false``.
``-fmad=false`` keeps every FP64 expression in the reference's evaluation
order with no fused multiply-add, which is what makes the FP64 path
bit-identical to the reference's arithmetic.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmf3d.so")
SOURCES = ["mf3d.cu", "topology.cpp"]
HEADERS = ["kernels.cuh", "coarse.cuh", "midcycle.cuh", "lmr.cuh", "outer.cuh", "server.cuh", "tecbin.cuh", "sip.cuh", "mf3d_internal.h", "../../include/mf3d.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [__file__]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-shared", "-o", OUT + ".tmp"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
