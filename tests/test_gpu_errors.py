"""Error paths and capacity growth on the GPU.

- A non-finite particle position stops the pass with DEM_ERR_STATE (the
  reference would run on with NaN). The cell hash clamps a NaN or infinite
  coordinate into the grid, and every later kernel of the pass returns on
  the abort word, so nothing is read or written out of bounds. A new state
  makes the context usable again.
- A grid with fewer than 3 cells along a periodic axis, where the
  reference's half shell lists one cell twice, is refused at creation.
- Candidate rows longer than their initial capacity of 32 grow, and the
  run stays bit-identical with the oracle."""
import numpy as np
import pytest

from dem3d_b200 import _abi
from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200.configs import DENSITY, KN, KT
from dem3d_b200.system import DEMError, DEMSystem
from tests.oracle_lib import oracle_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_nonfinite_position_is_a_state_error(bad):
    w = configs.settling(n=300, seed=2, sigma_v=0.5)
    g = DEMSystem(w.params)
    pos = w.pos.copy()
    pos[17, 2] = bad
    g.set_state(pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
    g.initialize_cell_distribution()
    with pytest.raises(DEMError) as e:
        g.run(1, 10)
    assert e.value.code == _abi.DEM_ERR_STATE
    # a new state clears the status words: the context runs on, exactly
    o = oracle_system(w.params)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
        s.initialize_cell_distribution()
        s.run(1, 30)
    a, b = g.get_state(), o.get_state()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_two_cells_on_a_periodic_axis_are_refused():
    prm = P.per_particle_params(density=DENSITY, kn=KN, kt=KT, en=0.8, et=0.8, mu=0.5, rmax=0.6,
                                lbox=(2.5, 2.5, 10.0), pbc=(True, True, False),
                                gravity=(0, 0, -1), time_step=1e-4)
    with pytest.raises(DEMError) as e:
        DEMSystem(prm)
    assert e.value.code == _abi.DEM_ERR_UNSUPPORTED


def test_long_candidate_rows_grow():
    """Large spheres among small ones (d 3 and 1) with the widest row skin
    (half of CutOff): a large sphere's row (the partners it meets as "i")
    holds about 55 candidates, past the initial capacity of 32."""
    w = configs.bidisperse_settling(n=3000, width=24.0, headroom=6.0, sigma_v=0.5,
                                    euler_intervals=10)
    g, o = DEMSystem(w.params), oracle_system(w.params)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
        s.initialize_cell_distribution()
    g.set_tuning(0.5, 0)
    for s in (g, o):
        s.run(1, 100)
    assert g.row_stats()["row_capacity"] > 48
    a, b = g.get_state(), o.get_state()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    ca, cb = g.get_contacts(), o.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    assert g.ncol() == o.ncol() > 0
