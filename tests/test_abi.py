"""The CUDA library loads and exports every entry point include/*.h declares.
(No compute call is made: there is no GPU in the CPU test environment.)"""
import ctypes as C
import glob
import os
import re

import pytest

from dem3d_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(dem_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_abi():
    names = declared_symbols()
    assert "dem_create" in names and "dem_move_particles" in names
    # the Python binding table covers every declared entry point
    assert set(names) <= set(_abi.all_symbols()) | {"dem_version"}


def test_library_exports_every_symbol():
    lib = _abi.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.dem_version().decode().startswith("dem3d_b200")


def test_no_silent_cpu_path_without_device():
    """Without a CUDA device dem_create fails loudly (DEM_ERR_NO_DEVICE)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dem3d_b200.configs import settling
    from dem3d_b200.system import DEMError, DEMSystem
    w = settling(n=10)
    with pytest.raises(DEMError) as ei:
        DEMSystem(w.params)
    assert ei.value.code == _abi.DEM_ERR_NO_DEVICE


def test_params_struct_layout():
    """ctypes mirror size equals the C struct size (checked with gcc)."""
    import subprocess
    import tempfile
    src = ('#include "%s"\n#include <stdio.h>\nint main(){printf("%%zu %%zu %%zu",'
           'sizeof(dem_params),sizeof(dem_wall),sizeof(dem_observables));}'
           % os.path.join(ROOT, "include", "dem3d_b200.h"))
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        subprocess.run(["gcc", c, "-o", os.path.join(d, "s")], check=True)
        out = subprocess.run([os.path.join(d, "s")], capture_output=True, text=True).stdout
    a, b, o = (int(x) for x in out.split())
    assert a == C.sizeof(_abi.DemParams)
    assert b == C.sizeof(_abi.DemWall)
    assert o == C.sizeof(_abi.DemObservables)
