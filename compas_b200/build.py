"""Build of the CUDA library libcompas_b200.so (sm_100a) in-tree.

The plain FP64 path must reproduce the reference's CPU arithmetic, so the library is compiled with
FMA contraction off (-fmad=false) and IEEE division and square root (the nvcc defaults).
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "csrc", "compas_b200.cu")
OUT = os.path.join(HERE, "libcompas_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-shared",
         "-I" + os.path.join(ROOT, "include")]


def sources() -> list:
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d))] + [os.path.join(ROOT, "include", "compas_b200.h")]


def build(force: bool = False, verbose: bool = False) -> str:
    newest = max(os.path.getmtime(s) for s in sources())
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        return OUT
    cmd = ["nvcc"] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", OUT, SRC]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)
