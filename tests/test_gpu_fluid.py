"""Fluid drag on the GPU (k_fluid_levels, k_fluid_drag, added in the pass
kernels) against the oracle.  The level sums run in a fixed tree instead of
index order, and CUDA's pow is not glibc's, so FP64 forces agree within the
1e-12 relative bound of the plain FP64 mode rather than bit for bit; a short
run stays within that drift."""
import numpy as np
import pytest

from dem3d_b200 import params as P
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system
from tests.test_fluid import fluid_case

pytestmark = pytest.mark.gpu


def _pair(w, fl, make_g=DEMSystem):
    g, o = make_g(w.params), oracle_system(w.params)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        s.set_fluid(fl)
    return g, o


def test_one_pass_forces_within_1e_12():
    w, fl = fluid_case(n=2000, flow=60.0)
    g, o = _pair(w, fl)
    for s in (g, o):
        s.compute_accelerations(update=False)
    a, b = g.get_state()["acc"], o.get_state()["acc"]
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())
    assert np.abs(b[:, 2] + 1.0).max() > 1e-3  # drag changes the accelerations


def test_run_with_drag_tracks_the_oracle():
    w, fl = fluid_case(n=2000, flow=60.0)
    g, o = _pair(w, fl)
    for s in (g, o):
        s.run(1, 120)  # Euler start-up, then graph replays with the fluid kernels
    a, b = g.get_state(), o.get_state()
    np.testing.assert_allclose(a["pos"], b["pos"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(a["vel"], b["vel"], rtol=0, atol=1e-7)
    ca, cb = g.get_contacts(), o.get_contacts()
    np.testing.assert_array_equal(ca["imin"], cb["imin"])
    np.testing.assert_array_equal(ca["imax"], cb["imax"])
    assert len(ca["imin"]) + len(ca["ip"]) > 0


def test_fluid_in_mixed_precision():
    w, fl = fluid_case(n=2000, flow=60.0)
    w.params.precision = P.PREC_MIXED
    g = DEMSystem(w.params)
    w.params.precision = P.PREC_FP64
    g64 = DEMSystem(w.params)
    for s in (g, g64):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        s.set_fluid(fl)
        s.compute_accelerations(update=False)
    a, b = g.get_state()["acc"], g64.get_state()["acc"]
    assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()
    g.run(1, 120)
    assert np.isfinite(g.get_state()["pos"]).all()
