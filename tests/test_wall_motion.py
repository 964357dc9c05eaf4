"""Moving walls (WallsInMovement, MoveWalls src/MDEM.f90:392-408) in the
oracle: the wall state after each kind of step is the closed form at the
step's Time, walls push the particles they touch, and stopping the motion
leaves the walls where they are."""
import math

import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from tests.oracle_lib import oracle_system


def closed_form(m, t):
    # MoveWalls at Time t, written out (Pi as the reference spells it)
    two_pi = 2.0 * 3.1415926535897932384626433832795
    pos, vel = [], []
    for k in range(3):
        ph = m["two_pi_frequency"][k] * t + m["phase_angle"][k]
        ph = ph - two_pi * float(int(ph / two_pi))
        pos.append(m["constant_factor"][k] + m["amplitude"][k] * math.cos(ph))
        vel.append(m["velocity_amplitude"][k] * math.sin(ph))
    return pos, vel


def floor_motion(w, amp=0.02, freq=20.0, phase=0.1):
    floor = w.params.walls[1]
    return P.wall_motion(list(floor.position), (0.0, 0.0, amp), (0.0, 0.0, freq),
                         (0.0, 0.0, phase))


def cone_motion(w):
    cone = w.params.walls[0]
    return P.wall_motion(list(cone.position), (0.01, 0.0, 0.03), (5.0, 0.0, 25.0),
                         (0.25, 0.0, 0.6))


def test_wall_motion_record_follows_the_input_reader():
    m = P.wall_motion((1.0, 2.0, 3.0), (0.5, 0.0, 0.25), (2.0, 0.0, 4.0), (0.25, 0.0, 0.5))
    two_pi = 2.0 * P.PI
    assert m["two_pi_frequency"] == [two_pi * 2.0, 0.0, two_pi * 4.0]
    assert m["velocity_amplitude"][0] == -two_pi * 2.0 * 0.5
    # at Time = 0 MoveWalls puts the wall back at its input position
    pos, _ = closed_form(m, 0.0)
    np.testing.assert_allclose(pos, (1.0, 2.0, 3.0), atol=1e-15)
    with pytest.raises(ValueError):
        P.wall_motion((0, 0, 0), (1, 1, 1), (-1.0, 0, 0), (0, 0, 0))


def test_walls_follow_movewalls_in_the_oracle():
    w = configs.hopper(n=120, seed=1006, euler_intervals=4)
    o = oracle_system(w.params)
    o.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
    o.initialize_cell_distribution()
    motion = [cone_motion(w), floor_motion(w)]
    start = o.walls()
    o.set_wall_motion(motion)
    np.testing.assert_array_equal(o.walls()["position"], start["position"])  # not moved yet
    dt = w.params.time_step
    o.move_particles_euler()  # Time advances by dt/4 four times
    t = 0.0
    for _ in range(4):
        t = t + dt / 4
    got = o.walls()
    for j, m in enumerate(motion):
        pos, vel = closed_form(m, t)
        assert list(got["position"][j]) == pos
        assert list(got["velocity"][j]) == vel
    for step in range(2, 40):
        o.move_particles(step)
    got = o.walls()
    for j, m in enumerate(motion):
        pos, vel = closed_form(m, 39 * dt)
        assert list(got["position"][j]) == pos
        assert list(got["velocity"][j]) == vel
    # stopping the motion keeps the walls where they are
    o.set_wall_motion(None)
    o.move_particles(40)
    np.testing.assert_array_equal(o.walls()["position"], got["position"])
    np.testing.assert_array_equal(o.walls()["velocity"], got["velocity"])


def test_a_rising_floor_lifts_a_resting_sphere():
    """One sphere on a floor that moves up: the contact force carries it."""
    w = configs.hopper(n=1, seed=1007, euler_intervals=4)
    floor_z = w.params.walls[1].position[2]
    pos = np.array([[0.0, 0.0, floor_z + 0.5 - 1e-3]])
    vel = np.zeros((1, 3))
    runs = []
    for amp in (0.0, 0.02):
        o = oracle_system(w.params)
        o.set_state(pos, vel, vel, comp=w.comp, radius=w.radius)
        o.initialize_cell_distribution()
        # phase 0.75: the floor starts at its rest height moving up at 2*pi*f*amp
        o.set_wall_motion([P.wall_motion((0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0)),
                           P.wall_motion(list(w.params.walls[1].position), (0.0, 0.0, amp),
                                         (0.0, 0.0, 5.0), (0.0, 0.0, 0.75))])
        o.run(1, 400)
        runs.append(o.get_state()["pos"][0, 2])
    assert runs[1] > runs[0] + 1e-3
