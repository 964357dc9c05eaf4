"""The reference's shipped example (examples/ball-bearings) on the GPU
against the oracle, bit for bit: spheres poured into an empty box (the
reference's generator), five cone walls orbiting on their circles, 45,000
steps through dem_run (graph chunks, pouring steps run one at a time, the
cone-wall kernels), until the 39 spheres touch each other and the cones."""
import numpy as np
import pytest

from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system
from tests.test_ball_bearings import start
from tests.test_particle_removal import export

pytestmark = pytest.mark.gpu


def test_ball_bearings_bit_exact():
    _, _, _, g = start(DEMSystem)
    _, _, _, o = start(oracle_system)
    g.run(1, 45000)
    o.run(1, 45000)
    assert g.n == o.n == 39
    a, b = export(g, True), export(o, True)
    for k in ("pos", "vel", "cell_index", "traversal", "cell_start", "prev"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in a["contacts"]:
        np.testing.assert_array_equal(a["contacts"][k], b["contacts"][k], err_msg=k)
    assert len(a["contacts"]["imin"]) > 0 and len(a["contacts"]["ip"]) > 0
    np.testing.assert_array_equal(g.walls()["position"], o.walls()["position"])
    assert g.rng() == o.rng() and g.ncol() == o.ncol()
