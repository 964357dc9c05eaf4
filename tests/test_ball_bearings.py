"""The reference's shipped example (examples/ball-bearings: five cone walls
orbiting at 1.5 Hz, steel spheres poured into an empty box) on the oracle:
its scaled parameters, and a run that pours, moves the walls on their
circles and settles spheres on the cones."""
import math

import numpy as np

from dem3d_b200 import configs
from tests.oracle_lib import oracle_system


def start(make, interval=0.01):
    w, motion, pour, seed = configs.ball_bearings(pouring_interval=interval)
    s = make(w.params)
    s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    s.initialize_cell_distribution()
    s.set_wall_motion(motion)
    s.set_pouring(pour)
    s.set_rng(dummy=seed)
    return w, motion, pour, s


def test_scaled_parameters():
    w, motion, pour, seed = configs.ball_bearings()
    p = w.params
    # LengthScale = the diameter (1 cm), 10 steps per collision time
    assert list(p.lbox) == [11.0, 11.0, 5.0] and p.comp_radius[0] == 0.5
    assert abs(p.time_step - 0.1) < 1e-6
    assert p.n_walls == 5 and all(p.walls[j].shape == 2 for j in range(5))
    assert [p.walls[j].l1 for j in range(5)] == [0.75, 0.0, 0.8, 0.0, 0.0]
    assert pour.target_number[0] == 39 and pour.max_attempts == 10 and pour.size[0] == 2.0
    # 0.5 s between attempts, in steps of 30 s / N
    assert pour.interval == round(0.5 / (30.0 / w.info["steps"]))
    assert seed == -20


def test_pouring_into_orbiting_cones():
    w, motion, pour, o = start(oracle_system)
    o.run(1, 30000)
    assert 25 <= o.n <= 39
    # the walls are where MoveWalls puts them at Time = 30000*dt
    t = 30000 * w.params.time_step
    two_pi = 2.0 * 3.1415926535897932384626433832795
    for j, m in enumerate(motion):
        for k in range(3):
            ph = m["two_pi_frequency"][k] * t + m["phase_angle"][k]
            ph = ph - two_pi * float(int(ph / two_pi))
            want = m["constant_factor"][k] + m["amplitude"][k] * math.cos(ph)
            assert o.walls()["position"][j][k] == want
    st = o.get_state()
    L = np.array(list(w.params.lbox))
    assert not np.any((st["pos"] > 0.5 * L) | (st["pos"] < -0.5 * L))
    assert o.count_contacts()[1] > 10  # spheres rest on the cone walls
