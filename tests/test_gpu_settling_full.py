"""The CPU-runnable settling configuration at full length, GPU against the
oracle bit for bit: 2,000 spheres (d = 1) settling onto a floor in a 10 x 10
periodic box, 20,000 ABM4 steps after the Euler start-up, through dem_run."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system

pytestmark = pytest.mark.gpu


def test_settling_2000_spheres_20000_steps():
    w = configs.settling()  # n = 2000, seed 1000, dt = 1e-4, e = 0.8, mu = 0.5
    g, o = DEMSystem(w.params), oracle_system(w.params)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        s.run(1, 20000)
    a, b = g.get_state(), o.get_state()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    ca, cb = g.get_contacts(), o.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    assert g.ncol() == o.ncol() > 0
    assert len(ca["ip"]) > 0  # the bed has reached the floor
