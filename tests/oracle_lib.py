"""Loads the CPU oracle (oracle/dem_oracle.c) behind the same ABI as the
CUDA library, for the tests to compare against (never as the product)."""
from __future__ import annotations

import ctypes as C
import os

from dem3d_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_CACHE = {}


def load_oracle(variant: str = "libdem_oracle.so") -> C.CDLL:
    if variant in _CACHE:
        return _CACHE[variant]
    import importlib.util
    spec = importlib.util.spec_from_file_location("oracle_build",
                                                  os.path.join(ROOT, "oracle", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    libs = mod.build()
    lib = C.CDLL(libs[variant])
    _abi.bind(lib, "orc_", _abi.SIGNATURES)
    lib.orc_set_literal_neighbour_cap.argtypes = [C.c_void_p, C.c_int32]
    lib.orc_set_literal_neighbour_cap.restype = C.c_int
    lib.orc_set_literal_removal.argtypes = [C.c_void_p, C.c_int32]
    lib.orc_set_literal_removal.restype = C.c_int
    _CACHE[variant] = lib
    return lib


def oracle_system(params, variant: str = "libdem_oracle.so"):
    from dem3d_b200.system import DEMSystem
    return DEMSystem(params, lib=load_oracle(variant), prefix="orc_")
