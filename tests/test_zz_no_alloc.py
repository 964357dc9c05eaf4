"""The allocation-free cell distribution against the context-based one.

dem_distribute_particles_noalloc exists for callers that may not allocate
device memory while they run (applications whose device memory all comes from
their own pool, services that forbid allocation after start-up because
cudaMalloc synchronises the device).  It must give exactly what
dem_initialize_cell_distribution gives -- the cell of every particle and every
cell's particles in list order -- on consecutive calls that reuse its one
static scratch array.  The inputs
and outputs here are device buffers owned by the test (torch tensors); the
entry point itself allocates nothing.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from dem3d_b200 import _abi, configs
from dem3d_b200.system import DEMSystem

pytestmark = pytest.mark.gpu


def context_cells(w):
    s = DEMSystem(w.params)
    s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
    s.initialize_cell_distribution()
    out = s.get_cells()
    s.close()
    return out


def noalloc_cells(lib, w):
    import torch
    n = w.n
    pos = torch.tensor(np.ascontiguousarray(w.pos), dtype=torch.float64, device="cuda")
    ci = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    tr = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    nx, ny, nz = DEMSystem(w.params).grid()
    cs = torch.full((nx * ny * nz + 1,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ncell = C.c_int32(0)
    err = C.create_string_buffer(256)
    st = lib.dem_distribute_particles_noalloc(C.byref(w.params), n, pos.data_ptr(), ci.data_ptr(),
                                              tr.data_ptr(), cs.data_ptr(), C.byref(ncell), None,
                                              err, 256)
    assert st == 0, err.value.decode()
    assert ncell.value == nx * ny * nz
    return ci.cpu().numpy(), tr.cpu().numpy(), cs.cpu().numpy()


def test_noalloc_matches_context_path_twice():
    lib = _abi.load_library()
    first = configs.settling(n=1500, seed=5)
    second = configs.dense_packing(n=8000, phi=0.55, seed=77, relax_steps=0)
    for w in (first, second):   # two calls in a row on the shared scratch array
        a = noalloc_cells(lib, w)
        b = context_cells(w)
        for x, y, name in zip(a, b, ("cell_index", "traversal", "cell_start")):
            np.testing.assert_array_equal(x, y, err_msg=name)


def test_noalloc_rejects_oversize():
    lib = _abi.load_library()
    w = configs.settling(n=10)
    err = C.create_string_buffer(256)
    st = lib.dem_distribute_particles_noalloc(C.byref(w.params), _abi.NOALLOC_MAX_PARTICLES + 1,
                                              None, None, None, None, None, None, err, 256)
    assert st == _abi.DEM_ERR_CAPACITY
    assert b"DEM_NOALLOC_MAX_PARTICLES" in err.value
