"""Spatial decomposition of one system into z-slabs, emulated on one GPU.

Every slab is its own context (its own arrays of every particle), advances
only the particles of its cell layers, and exchanges with its neighbours
through packed device buffers copied between the contexts (the same
buffers a multi-GPU run sends between ranks).  The composed state (each
particle from the slab that owns it) must equal the undivided system's
bit for bit: same sweep contributions in the same order, same history
records, same cell lists, same migrations."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200 import slab as S
from dem3d_b200.system import DEMError, DEMSystem
from tests.test_gpu_scale import transfer

pytestmark = pytest.mark.gpu


def _base(precision, n=64_000, seed=1021):
    w = configs.dense_packing(n=n, phi=0.55, seed=seed, tile=8000)
    w.params.precision = precision
    w.params.hist_capacity = 16
    g = DEMSystem(w.params)
    g.set_state(w.pos, w.vel, w.omega, radius=w.radius)
    g.initialize_cell_distribution()
    g.run(1, 20)
    return w, g


def _slabs(w, g, nslabs):
    nz = g.grid()[2]
    ranges = S.slab_ranges(nz, nslabs)
    slabs = []
    for z0, z1 in ranges:
        s = DEMSystem(w.params)
        transfer(g, s, radius=w.radius)
        s.slab_set_range(z0, z1)
        slabs.append(s)
    return slabs, ranges


@pytest.mark.parametrize("nslabs,precision", [(2, P.PREC_FP64), (3, P.PREC_FP64),
                                              (4, P.PREC_MIXED)])
def test_slabs_equal_the_whole_system(nslabs, precision):
    w, g = _base(precision)
    ref = DEMSystem(w.params)
    transfer(g, ref, radius=w.radius)
    slabs, ranges = _slabs(w, g, nslabs)
    ncol0 = g.ncol()
    steps = range(21, 61)
    tr = S.LocalTransport(slabs, periodic=True, cap_bytes=64 << 20)
    for step in steps:
        S.move_particles(tr, step)
    ref.run(steps[0], steps[-1])
    want = ref.get_state()
    got = S.compose_state(slabs)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=f"{nslabs} slabs: {k}")
    assert ncol0 + sum(s.ncol() - ncol0 for s in slabs) == ref.ncol()
    # particles did cross slab boundaries, and the exchanges carried data
    owned = [s.slab_owned() for s in slabs]
    assert sum(int(o.sum()) for o in owned) == g.n
    assert tr.bytes_moved > 0
    assert ref.count_contacts()[0] > 0


def test_slab_migration_under_fast_motion():
    """Fast particles (σ_v = 20, 2e-3 per pass): hundreds cross the slab
    boundaries in 60 steps, with their rings and history records."""
    w = configs.dense_packing(n=64_000, phi=0.55, seed=1022, tile=8000)
    w.params.hist_capacity = 16
    vel = np.random.default_rng(5).normal(0.0, 20.0, w.vel.shape)
    g = DEMSystem(w.params)
    g.set_state(w.pos, vel, w.omega, radius=w.radius)
    g.initialize_cell_distribution()
    g.run(1, 8)
    ref = DEMSystem(w.params)
    transfer(g, ref, radius=w.radius)
    slabs, ranges = _slabs(w, g, 2)
    before = [s.slab_owned() for s in slabs]
    tr = S.LocalTransport(slabs, periodic=True, cap_bytes=64 << 20)
    for step in range(9, 69):
        S.move_particles(tr, step)
    ref.run(9, 68)
    want = ref.get_state()
    got = S.compose_state(slabs)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    after = [s.slab_owned() for s in slabs]
    moved = int(np.count_nonzero(before[0] != after[0]))
    assert moved > 100, moved


def test_slab_range_is_checked():
    w, g = _base(P.PREC_FP64, n=8000, seed=1023)
    nz = g.grid()[2]
    for z0, z1 in ((0, 0), (-1, 3), (0, nz + 1), (2, 3)):
        with pytest.raises(DEMError):
            g.slab_set_range(z0, z1)


def test_slabs_over_a_floor_equal_the_whole_system():
    """A bed over a floor wall (z not periodic: the slabs form a chain, the
    bottom slab holds the wall contacts and their records), spheres moving
    fast enough (σ_v = 5, dt = 5e-4) to cross slab boundaries with their
    wall records."""
    w = configs.settling(n=4096, layer_side=16, seed=1024, dt=5e-4, sigma_v=5.0, gravity=10.0,
                         headroom=8.0, euler_intervals=10)
    w.params.hist_capacity = 16
    g = DEMSystem(w.params)
    g.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    g.initialize_cell_distribution()
    g.run(1, 12)
    nz = g.grid()[2]
    nslabs = 3 if nz >= 6 else 2
    ref = DEMSystem(w.params)
    transfer(g, ref, comp=w.comp)
    slabs = []
    for z0, z1 in S.slab_ranges(nz, nslabs):
        s = DEMSystem(w.params)
        transfer(g, s, comp=w.comp)
        s.slab_set_range(z0, z1)
        slabs.append(s)
    before = [s.slab_owned() for s in slabs]
    tr = S.LocalTransport(slabs, periodic=False, cap_bytes=64 << 20)
    for step in range(13, 413):
        S.move_particles(tr, step)
    ref.run(13, 412)
    want = ref.get_state()
    got = S.compose_state(slabs)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    ncol0 = g.ncol()
    assert ncol0 + sum(s.ncol() - ncol0 for s in slabs) == ref.ncol()
    assert ref.count_contacts()[1] > 0  # spheres on the floor
    after = [s.slab_owned() for s in slabs]
    assert int(np.count_nonzero(before[0] != after[0])) > 20
