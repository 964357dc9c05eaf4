"""Build recipe for the CPU oracle (test infrastructure only).

``libdem_oracle.so``      -O2 -ffp-contract=off: the oracle the tests compare against.
``libdem_oracle_fast.so`` -O3 -ffp-contract=off: the same code built with the
                          reference Makefile's optimisation level, timed as the
                          CPU baseline (portable ISA; the bench may rebuild it
                          with -march=native on the host it runs on).
No Fortran compiler exists in this environment, so the reference itself cannot
be built: ``oracle/_ref`` stays empty.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "build")
SRC = os.path.join(HERE, "dem_oracle.c")
HDR = os.path.join(HERE, "..", "include", "dem3d_b200.h")
VARIANTS = {
    "libdem_oracle.so": ["-O2", "-ffp-contract=off"],
    "libdem_oracle_fast.so": ["-O3", "-ffp-contract=off"],
}


def build(force: bool = False, native_dir: str | None = None) -> dict[str, str]:
    os.makedirs(BUILD, exist_ok=True)
    out = {}
    for name, flags in VARIANTS.items():
        lib = os.path.join(BUILD, name)
        fresh = os.path.exists(lib) and all(
            os.path.getmtime(d) <= os.path.getmtime(lib) for d in (SRC, HDR))
        if force or not fresh:
            subprocess.run(["gcc", "-std=c11", "-fPIC", "-shared", *flags, SRC, "-o", lib, "-lm"],
                           check=True)
        out[name] = lib
    if native_dir:
        lib = os.path.join(native_dir, "libdem_oracle_native.so")
        subprocess.run(["gcc", "-std=c11", "-fPIC", "-shared", "-O3", "-march=native",
                        "-ffp-contract=off", SRC, "-o", lib, "-lm"], check=True)
        out["libdem_oracle_native.so"] = lib
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
