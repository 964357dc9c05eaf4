"""Ensembles: many independent systems in one context (dem_create_ensemble).

Every stage of a step runs as one launch over all systems, with per-system
cell grids, boxes, walls and materials.  Within a system the global
numbering is an offset shift of the system's own numbering, so every
ordering rule of the reference is unchanged.  An ensemble must therefore
reproduce, bit for bit, each of its systems run alone in its own context
(which the parity tests pin to the oracle)."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200.system import DEMSystem

pytestmark = pytest.mark.gpu


def small_ensemble(precision, seed=7):
    # uneven sizes, per-system friction and restitution; fast particles so
    # that many change cell and collide within a few dozen steps
    return configs.settling_ensemble(n_systems=5, nmin=100, nmax=700, seed=seed, sigma_v=4.0,
                                     precision=precision, euler_intervals=10)


def run_ensemble(e, steps):
    s = DEMSystem.ensemble(e.params, e.counts)
    s.set_state(e.pos, e.vel, e.omega, radius=e.radius)
    s.initialize_cell_distribution()
    s.run(1, steps)
    out = s.get_state(), s.get_contacts(), s.ncol()
    s.close()
    return out


def run_alone(e, k, steps):
    prm, pos, vel, om, rad = e.system(k)
    s = DEMSystem(prm)
    s.set_state(pos, vel, om, radius=rad)
    s.initialize_cell_distribution()
    s.run(1, steps)
    out = s.get_state(), s.get_contacts(), s.ncol()
    s.close()
    return out


@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_MIXED])
def test_ensemble_equals_systems_run_alone(precision):
    e = small_ensemble(precision)
    steps = 60
    st, ct, ncol = run_ensemble(e, steps)
    off = np.concatenate([[0], np.cumsum(e.counts)])
    total_ncol = 0
    pairs = 0
    for k in range(len(e.counts)):
        a, b = off[k], off[k + 1]
        st1, ct1, ncol1 = run_alone(e, k, steps)
        for key in st1:
            np.testing.assert_array_equal(st[key][a:b], st1[key], err_msg=f"system {k} {key}")
        sel = (ct["imin"] >= a) & (ct["imin"] < b)
        np.testing.assert_array_equal(ct["imin"][sel] - a, ct1["imin"], err_msg=f"system {k}")
        np.testing.assert_array_equal(ct["imax"][sel] - a, ct1["imax"], err_msg=f"system {k}")
        np.testing.assert_array_equal(ct["ft"][sel], ct1["ft"], err_msg=f"system {k}")
        wsel = (ct["ip"] >= a) & (ct["ip"] < b)
        np.testing.assert_array_equal(ct["ip"][wsel] - a, ct1["ip"], err_msg=f"system {k}")
        np.testing.assert_array_equal(ct["ftw"][wsel], ct1["ftw"], err_msg=f"system {k}")
        total_ncol += ncol1
        pairs += len(ct1["imin"])
    assert ncol == total_ncol
    assert pairs > 0  # the systems do collide


def test_ensemble_rejects_mismatched_integrators():
    e = small_ensemble(P.PREC_FP64)
    e.params[1].time_step = e.params[0].time_step * 2
    with pytest.raises(Exception):
        DEMSystem.ensemble(e.params, e.counts)


def test_ensemble_rejects_moving_walls():
    e = small_ensemble(P.PREC_FP64)
    s = DEMSystem.ensemble(e.params, e.counts)
    with pytest.raises(Exception):
        s.set_wall_motion([P.wall_motion((0, 0, 0), (0, 0, 0.1), (0, 0, 1.0), (0, 0, 0))])
    s.close()
