"""Storage in cell order (dem_set_reorder) changes where particles are
stored, never a result.

Every stored particle number is renamed with the permutation, the
reference's numbering is kept for the one step rule that depends on it (a
cell's arrivals enter its list in decreasing index), and every call that
reads or writes particle data first restores the reference's order.  A run
that reorders every few steps must therefore equal the same run without
reordering bit for bit: states, contact records, cell lists, Ncol."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system
from tests.test_particle_removal import export

pytestmark = pytest.mark.gpu


def _same(a, b, what):
    sa, sb = a.get_state(), b.get_state()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=f"{what} {k}")
    ca, cb = a.get_contacts(), b.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=f"{what} {k}")
    for x, y in zip(a.get_cells(), b.get_cells()):
        np.testing.assert_array_equal(x, y, err_msg=f"{what} cells")
    assert a.ncol() == b.ncol(), what


def _dense(precision, sigma_v=3.0):
    w = configs.dense_packing(n=64_000, phi=0.55, seed=1031, tile=8000)
    w.params.precision = precision
    vel = np.random.default_rng(9).normal(0.0, sigma_v, w.vel.shape)
    s = DEMSystem(w.params)
    s.set_state(w.pos, vel, w.omega, radius=w.radius)
    s.initialize_cell_distribution()
    return s


@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_MIXED])
def test_reordered_dense_run_is_bit_identical(precision):
    a, b = _dense(precision), _dense(precision)
    b.set_reorder(12)
    a.run(1, 200)
    b.run(1, 200)
    assert b.reorder()["reorders"] >= 10
    _same(a, b, "dense")
    # a state read in the middle, then more steps (restore, then permute again)
    a.run(201, 260)
    b.run(201, 260)
    _same(a, b, "dense, continued")


def test_reordered_bed_with_walls_equals_the_oracle():
    """Two components, a floor and side walls (wall records move with their
    spheres), reordered every 8 steps, against the oracle."""
    w = configs.bidisperse_settling(n=3000, width=24.0, headroom=6.0, sigma_v=0.5)
    g, o = DEMSystem(w.params), oracle_system(w.params)
    g.set_reorder(8)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
        s.initialize_cell_distribution()
        s.run(1, 400)
    _same(g, o, "bidisperse")
    assert g.reorder()["reorders"] > 20


def test_reordered_ensemble_and_persistent_chunks():
    e = configs.settling_ensemble(n_systems=6, nmin=100, nmax=900, seed=11, sigma_v=4.0,
                                  euler_intervals=10)
    out = []
    for reorder, mode in ((0, 0), (8, 0), (8, 1)):
        s = DEMSystem.ensemble(e.params, e.counts)
        s.set_launch_shape(launch_mode=mode)
        s.set_reorder(reorder)
        s.set_state(e.pos, e.vel, e.omega, radius=e.radius)
        s.initialize_cell_distribution()
        s.run(1, 83)
        out.append(s)
    _same(out[0], out[1], "ensemble, graph chunks")
    _same(out[0], out[2], "ensemble, persistent chunks")


def test_reordered_discharge_and_pouring():
    """Removals and insertions in a reordered run (each restores the
    reference's order first), against the oracle."""
    w = configs.discharge(d_out=5.0, mu=0.2)
    g, o = DEMSystem(w.params), oracle_system(w.params)
    g.set_reorder(16)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        s.run(1, 800)
    assert g.n == o.n < w.pos.shape[0]
    a, b = export(g, True), export(o, True)
    for k in ("pos", "vel", "cell_index", "traversal", "cell_start", "prev"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert g.ncol() == o.ncol()
    from tests.test_pouring import filling_box, start
    prm, pos, comp, pour = filling_box(interval=4)
    g = start(DEMSystem, prm, pos, comp, pour)
    o = start(oracle_system, prm, pos, comp, pour)
    g.set_reorder(10)
    g.run(1, 400)
    o.run(1, 400)
    assert g.n == o.n > pos.shape[0]
    sa, sb = g.get_state(), o.get_state()
    for k in sb:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=f"pouring {k}")
