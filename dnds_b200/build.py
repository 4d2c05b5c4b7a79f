"""Builds libdndsg.so (the sm_100a CUDA library behind include/dndsg.h) in-tree."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdndsg.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("dndsg.cu", "dndsg_bodies.cuh", "dndsg_math.cuh", "dndsg_limiter.cuh",
                                                         "dndsg_mlp.cuh", "dndsg_sa.cuh", "dndsg_dual.cuh", "dndsg_async.cuh")]
HEADERS = [os.path.join(ROOT, "include", "dndsg.h")]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --prec-div/--prec-sqrt=false relax single-precision division and square root only
# (the FP32-bulk flux); double precision is unaffected
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-shared", "--expt-relaxed-constexpr",
         "--prec-div=false", "--prec-sqrt=false"]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [NVCC, *ARCH, *FLAGS, "-o", LIB + ".tmp", os.path.join(HERE, "csrc", "dndsg.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
