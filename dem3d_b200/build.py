"""Build recipe for the sm_100a shared library ``libdem3d_b200.so``.

The library is compiled in-tree with nvcc (static CUDA runtime, so the .so
only needs the driver at run time).  ``dem_lib.cu`` holds the FP64 path and is
compiled with ``-fmad=false``: the exact path must not fuse multiply-adds,
which is what makes it bit-identical to the reference arithmetic.  The
mixed-precision kernels (``dem_mixed.cu``) use the hardware's approximate FP32
division and square root, and are compiled with ``-fmad=false`` too: with
contraction left to the compiler, the same expression can be fused in one
kernel and not in another that inlines the same code (the persistent chunk
kernel), and the two launch modes would then differ in the last bits.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdem3d_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills"]
# dem_mixed.cu: FP32 contact arithmetic within a stated 1e-5 tolerance, so
# division and square root may use the hardware approximations (~1 ulp); no
# contraction, so that every kernel that inlines the same code rounds alike
SOURCES = [("dem_lib.cu", ["-fmad=false", "-Xcompiler", "-ffp-contract=off"]),
           ("dem_mixed.cu", ["-fmad=false", "--prec-div=false", "--prec-sqrt=false"])]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdem3d_b200.so")


def _deps() -> list[str]:
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    out.append(os.path.join(HERE, "..", "include", "dem3d_b200.h"))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src, flags in SOURCES:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *COMMON, *flags, *(extra or []), "-c", os.path.join(CSRC, src),
               "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", *objs, "-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
