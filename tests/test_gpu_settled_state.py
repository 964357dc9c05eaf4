"""The predictor pass leaves Particle a, alpha in its ABM ring slot and
Predicted x (FP64 mode: v, w too) in the pass copies; the calls that read or
change particle data write them back first.  These runs interleave such
calls with graph-replayed steps and compare everything with the oracle bit
for bit (FP64): exports straight after a run, an upload of positions and
velocities only (a and alpha stay where the predictor left them), a round
trip of the ABM ring, a single force pass and an Euler start-up step after
ABM steps (its ring store reads Particle a, alpha)."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system

pytestmark = pytest.mark.gpu


def _pair(w):
    g = DEMSystem(w.params)
    o = oracle_system(w.params)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
        s.initialize_cell_distribution()
    return g, o


def _same(g, o, what):
    for name, get in (("state", "get_state"), ("predicted", "get_predicted")):
        a, b = getattr(g, get)(), getattr(o, get)()
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what}: {name}.{k}")
    # the ring in logical order, Previous(ipc(k)) (the library's physical
    # slots may be numbered differently)
    np.testing.assert_array_equal(g.logical_ring(), o.logical_ring(), err_msg=f"{what}: ring")


def test_exports_and_partial_uploads_between_runs():
    w = configs.settling(n=600, seed=11, sigma_v=0.5)
    g, o = _pair(w)
    try:
        for s in (g, o):
            s.run(1, 40)
        _same(g, o, "after the first run")
        # positions, velocities and angular velocities only: a and alpha
        # are not touched by the upload
        st = o.get_state()
        for s in (g, o):
            s.update_state(pos=st["pos"], vel=st["vel"], omega=st["omega"])
            s.run(41, 80)
        _same(g, o, "after an upload without accelerations")
        # the ring read and written back as it is
        prev, ipc = o.get_integration()
        for s in (g, o):
            s.set_integration(prev, ipc)
            s.run(81, 120)
        _same(g, o, "after a ring round trip")
    finally:
        g.close()
        o.close()


def test_force_pass_and_euler_step_after_abm_steps():
    w = configs.settling(n=500, seed=12, sigma_v=0.5)
    g, o = _pair(w)
    try:
        for s in (g, o):
            s.run(1, 30)
            s.compute_accelerations(use_predicted=True, update=False)
        _same(g, o, "after a force pass on Predicted")
        for s in (g, o):
            s.move_particles_euler()
            s.run(31, 60)
        _same(g, o, "after an Euler step between ABM steps")
    finally:
        g.close()
        o.close()
