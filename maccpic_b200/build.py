"""Build libem2g.so in-tree with nvcc for sm_100a.

``python -m maccpic_b200.build`` compiles every ``csrc/*.cu`` to an object
under ``maccpic_b200/_build/`` and links ``maccpic_b200/libem2g.so``.
Objects are rebuilt when their source or any header is newer.

The FP64 drop-in kernels (``push_f64.cu``, ``fields_f64.cu`` and the others in
``NO_FMA``) are compiled
with ``-fmad=false`` so that each product and sum is rounded separately, as
em2's gfortran build does on x86-64; the FP32 kernels keep FMA contraction.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libem2g.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
NO_FMA = {"push_f64.cu", "push_fast_f64.cu", "fields_f64.cu", "smooth2_static.cu", "setv.cu"}


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def build(verbose: bool = False, extra_flags=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_time = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    objs = []
    changed = False
    for src in sources:
        name = os.path.basename(src)
        obj = os.path.join(BUILD, name[:-3] + ".o")
        objs.append(obj)
        if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hdr_time):
            continue
        flags = list(COMMON) + (["-fmad=false"] if name in NO_FMA else [])
        flags += list(extra_flags or [])
        cmd = [NVCC] + ARCH + flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        changed = True
    if changed or not os.path.exists(LIB) or any(
            os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
