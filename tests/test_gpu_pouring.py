"""Pouring on the GPU (candidate points tested by k_pour_test, k_insert)
against the oracle: the same spheres go in at the same steps and places, the
generator ends in the same state, and the trajectories stay bit-identical,
whether the arrays had room reserved at dem_set_state or grow on the way."""
import numpy as np
import pytest

from dem3d_b200 import _abi
from dem3d_b200 import params as P
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system
from tests.test_particle_removal import export
from tests.test_pouring import filling_box, start

pytestmark = pytest.mark.gpu


def _same(g, o, what):
    a, b = export(g, True), export(o, True)
    for k in ("pos", "vel", "cell_index", "traversal", "cell_start", "prev"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what} {k}")
    for k in a["contacts"]:
        np.testing.assert_array_equal(a["contacts"][k], b["contacts"][k], err_msg=f"{what} {k}")
    np.testing.assert_array_equal(g.comp, o.comp, err_msg=what)
    assert g.rng() == o.rng(), what
    assert g.ncol() == o.ncol(), what


@pytest.mark.parametrize("shape", [_abi.POUR_RECTANGLE, _abi.POUR_CIRCLE])
def test_pouring_run_bit_exact(shape):
    prm, pos, comp, pour = filling_box(shape=shape, interval=4)
    g = start(DEMSystem, prm, pos, comp, pour)
    o = start(oracle_system, prm, pos, comp, pour)
    g.run(1, 700)
    o.run(1, 700)
    assert g.n == o.n > pos.shape[0] + 10
    _same(g, o, "pouring")


def test_capacity_reserved_or_grown_gives_the_same_run():
    """Pouring set before dem_set_state reserves the rows up front; set after
    it, the arrays grow (contents moved, rows and prepared copies rebuilt)."""
    prm, pos, comp, pour = filling_box(interval=3)
    a = DEMSystem(prm)
    a.set_pouring(pour)
    a.set_state(pos, np.zeros_like(pos), np.zeros_like(pos), comp=comp)
    a.initialize_cell_distribution()
    a.set_rng(dummy=-7)
    b = DEMSystem(prm)
    b.set_state(pos, np.zeros_like(pos), np.zeros_like(pos), comp=comp)
    b.initialize_cell_distribution()
    b.run(1, 20)  # a few steps without pouring, then the arrays grow mid-run
    b.set_pouring(pour)
    b.set_rng(dummy=-7)
    a.set_pouring(None)
    a.run(1, 20)
    a.set_pouring(pour)
    o = oracle_system(prm)
    o.set_state(pos, np.zeros_like(pos), np.zeros_like(pos), comp=comp)
    o.initialize_cell_distribution()
    o.run(1, 20)
    o.set_pouring(pour)
    o.set_rng(dummy=-7)
    for s in (a, b, o):
        s.run(21, 400)
    assert a.n == b.n == o.n > pos.shape[0]
    _same(a, o, "reserved")
    _same(b, o, "grown")


def test_pouring_mixed_precision_runs():
    prm, pos, comp, pour = filling_box(interval=4)
    prm.precision = _abi.PREC_MIXED
    g = start(DEMSystem, prm, pos, comp, pour)
    g.run(1, 700)
    assert g.n > pos.shape[0] + 10
    assert np.isfinite(g.get_state()["pos"]).all()
    counts = np.bincount(g.comp, minlength=2)
    assert counts[0] <= 60 and counts[1] <= 45
