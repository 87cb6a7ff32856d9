"""Build of the CUDA library libcompas_b200.so (sm_100a) in-tree.

The plain FP64 path must reproduce the reference's CPU arithmetic, so the library is compiled with
FMA contraction off (-fmad=false) and IEEE division and square root (the nvcc defaults). The mixed
form keeps contraction off too: its FMAs are written out (__fmaf_rn) where they are wanted, so every
launch shape of a stage kernel gives the same bits (with contraction on, the compiler contracted the
launch shapes' instantiations differently, and it measured no faster). The stage kernels of each
model and dimension are separate translation units per precision form (csrc/kern_<model>.cu plain
FP64, csrc/kern_<model>_mixed.cu mixed precision), compiled in parallel and linked with the C-ABI
unit (csrc/compas_b200.cu).
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libcompas_b200.so")
OBJ = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]


def units() -> list:
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]


def sources() -> list:
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))] + [os.path.join(ROOT, "include", "compas_b200.h")]


def build(force: bool = False, verbose: bool = False) -> str:
    newest = max(os.path.getmtime(s) for s in sources())
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    objs, procs = [], []
    for u in units():
        o = os.path.join(OBJ, os.path.basename(u)[:-3] + ".o")
        objs.append(o)
        cmd = ["nvcc"] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", "-o", o, u]
        procs.append((u, subprocess.Popen(cmd)))
    failed = [u for u, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc " + " ".join(failed))
    subprocess.check_call(["nvcc"] + ARCH + ["-shared", "-o", OUT] + objs)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)
