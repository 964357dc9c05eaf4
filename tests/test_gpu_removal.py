"""UpdateParticleList on the GPU (k_escape_list + k_remove) against the
oracle: the same particles leave, the last particle takes each one's place,
and cell lists, contact records and the ABM ring come out bit-identical;
dem_run removes after every step, inside captured chunks too."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system
from tests.test_particle_removal import dense_case, export, picks_near_last, push_out

pytestmark = pytest.mark.gpu


def _same_exports(a, b, what):
    for k in ("pos", "vel", "cell_index", "traversal", "cell_start", "prev"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what} {k}")
    for k in a["contacts"]:
        np.testing.assert_array_equal(a["contacts"][k], b["contacts"][k], err_msg=f"{what} {k}")


def test_gpu_removal_equals_oracle():
    w, g = dense_case(DEMSystem)
    _, o = dense_case(oracle_system)
    n = g.n
    picks = picks_near_last(o, n)
    for s in (g, o):
        push_out(s, w, picks)
    _same_exports(export(g, True), export(o, True), "before")
    assert g.update_particle_list() == o.update_particle_list() == 3
    assert g.n == o.n == n - 3
    _same_exports(export(g, True), export(o, True), "after removal")
    assert g.removal_stats() == o.removal_stats()
    assert g.removal_stats()["records_moved"] > 0
    for s in (g, o):
        s.run(13, 40)
    _same_exports(export(g, True), export(o, True), "after 28 more steps")
    assert g.ncol() == o.ncol()


def _discharge(make, **kw):
    w = configs.discharge(d_out=5.0, mu=0.2, **kw)
    s = make(w.params)
    s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    s.initialize_cell_distribution()
    return w, s


@pytest.mark.parametrize("capacity", [16, 1])
def test_discharge_bit_exact(capacity):
    """Spheres leave a hopper through the bottom of the box for 800 steps:
    removals inside graph replays stop the chunk before the next step; with
    tables of one record per particle, removals also grow the tables."""
    w = configs.discharge(d_out=5.0, mu=0.2)
    w.params.hist_capacity = capacity
    g, o = DEMSystem(w.params), oracle_system(w.params)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        s.run(1, 800)
    assert g.n == o.n < w.pos.shape[0]
    _same_exports(export(g, True), export(o, True), "discharge")
    assert g.ncol() == o.ncol()
    assert g.removal_stats() == o.removal_stats()
    np.testing.assert_array_equal(g.comp, o.comp)


def test_discharge_mixed_precision_runs():
    w, g = _discharge(DEMSystem, precision=P.PREC_MIXED)
    g.run(1, 800)
    assert g.n < w.pos.shape[0]
    st = g.get_state()
    L = np.array(list(w.params.lbox))
    assert np.isfinite(st["pos"]).all()
    assert not np.any((st["pos"] > 0.5 * L) | (st["pos"] < -0.5 * L))
    ct = g.get_contacts()
    assert ct["imin"].max(initial=-1) < g.n and ct["ip"].max(initial=-1) < g.n
