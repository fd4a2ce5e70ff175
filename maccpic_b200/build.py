"""Build libem2g.so in-tree with nvcc for sm_100a.

``python -m maccpic_b200.build`` compiles every ``csrc/*.cu`` to an object
under ``maccpic_b200/_build/`` and links ``maccpic_b200/libem2g.so``
(``--checked`` also links ``libem2g_checked.so``, the bounds-checked build).
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
# The bounds-checked library (libem2g_checked.so): the same objects, except
# that the units holding the FP32 push are compiled with -DEM2G_BOUNDS_CHECK
# (every index checked before its access, a miss counted and skipped).
CHECKED = {"push_fast_f32.cu", "ens_step.cu"}
BUILD_CHECKED = os.path.join(PKG, "_build_checked")
LIB_CHECKED = os.path.join(PKG, "libem2g_checked.so")


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _compile(src: str, obj: str, flags, hdr_time: float, verbose: bool) -> bool:
    if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= hdr_time):
        return False
    cmd = [NVCC] + ARCH + list(flags) + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return True


def _link(lib: str, objs, changed: bool, verbose: bool) -> None:
    if changed or not os.path.exists(lib) or any(
            os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + list(objs) + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


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
        flags = list(COMMON) + (["-fmad=false"] if name in NO_FMA else [])
        flags += list(extra_flags or [])
        changed |= _compile(src, obj, flags, hdr_time, verbose)
    _link(LIB, objs, changed, verbose)
    return LIB


def build_checked(verbose: bool = False) -> str:
    """libem2g_checked.so: the ordinary objects, with the FP32 push's units
    compiled with -DEM2G_BOUNDS_CHECK."""
    build(verbose=verbose)
    os.makedirs(BUILD_CHECKED, exist_ok=True)
    hdr_time = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    objs = []
    changed = False
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        name = os.path.basename(src)
        if name not in CHECKED:
            objs.append(os.path.join(BUILD, name[:-3] + ".o"))
            continue
        obj = os.path.join(BUILD_CHECKED, name[:-3] + ".o")
        objs.append(obj)
        flags = list(COMMON) + ["-DEM2G_BOUNDS_CHECK"]
        changed |= _compile(src, obj, flags, hdr_time, verbose)
    _link(LIB_CHECKED, objs, changed, verbose)
    return LIB_CHECKED


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
    if "--checked" in sys.argv:
        print(build_checked(verbose="-v" in sys.argv))
