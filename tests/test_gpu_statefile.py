"""Checkpoint/resume on the GPU through the reference's state-file layout:
a run stopped after step k, saved, read back into a new context and run on
is bit-identical with the uninterrupted run and with the oracle, and a state
file written from the oracle resumes on the GPU."""
import os

import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200 import statefile as SF
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system

pytestmark = pytest.mark.gpu


def _start(make, w, motion):
    s = make(w.params)
    s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
    s.initialize_cell_distribution()
    if motion:
        s.set_wall_motion(motion)
    return s


def _vibration(w):
    cone, floor = w.params.walls[0], w.params.walls[1]
    return [P.wall_motion(list(cone.position), (0.01, 0.0, 0.03), (5.0, 0.0, 25.0),
                          (0.25, 0.0, 0.6)),
            P.wall_motion(list(floor.position), (0.0, 0.0, 0.02), (0.0, 0.0, 20.0),
                          (0.0, 0.0, 0.1))]


def _save(system, w, step, path):
    comps = SF.component_records([P.Component(len(w.pos), 1.0, configs.DENSITY,
                                              2.0 * configs.KN, 2.0 * configs.KT)])
    st = SF.capture(system, components=comps,
                    wall_stiffness=[(2.0 * configs.KN, 2.0 * configs.KT)] * 2, step=step)
    SF.write_state(path, st)
    return SF.read_state(path, w.params.method_order - 1)


def _same(a, b, what):
    sa, sb = a.get_state(), b.get_state()
    for k in ("pos", "vel", "omega"):
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=f"{what} {k}")
    ca, cb = a.get_contacts(), b.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=f"{what} {k}")
    for x, y in zip(a.get_cells(), b.get_cells()):
        np.testing.assert_array_equal(x, y, err_msg=what)
    assert a.ncol() == b.ncol(), what


@pytest.mark.parametrize("moving", [False, True])
def test_gpu_resume_is_bit_identical(tmp_path, moving):
    w = configs.hopper(n=600, seed=1005)
    motion = _vibration(w) if moving else None
    full = _start(DEMSystem, w, motion)
    full.run(1, 700)
    part = _start(DEMSystem, w, motion)
    part.run(1, 333)
    back = _save(part, w, 333, os.path.join(tmp_path, "g.stt"))
    res = DEMSystem(SF.params_with_walls(w.params, back))
    if motion:
        res.set_wall_motion(motion)
    first = SF.restore(res, back)
    assert first == 334
    res.run(first, 700)
    _same(full, res, "gpu resume")
    o = _start(oracle_system, w, motion)
    o.run(1, 700)
    _same(full, o, "gpu vs oracle")


def test_oracle_state_file_resumes_on_the_gpu(tmp_path):
    """Interoperability: the file written from the oracle run continues on the
    GPU exactly as the oracle continues."""
    w = configs.bidisperse_settling(n=3000, width=24.0, headroom=6.0, sigma_v=0.5,
                                    euler_intervals=10)
    o = _start(oracle_system, w, None)
    o.run(1, 200)
    comps = SF.component_records(
        [P.Component(int(np.count_nonzero(w.comp == k)), d, configs.DENSITY, 2.0 * configs.KN,
                     2.0 * configs.KT) for k, d in enumerate((1.0, 3.0))])
    st = SF.capture(o, components=comps, wall_stiffness=[(2.0 * configs.KN, 2.0 * configs.KT)] * 5,
                    step=200)
    path = os.path.join(tmp_path, "o.stt")
    SF.write_state(path, st)
    back = SF.read_state(path, w.params.method_order - 1)
    g = DEMSystem(SF.params_with_walls(w.params, back))
    first = SF.restore(g, back)
    g.run(first, 400)
    o.run(201, 400)
    _same(o, g, "oracle file on gpu")


def test_gpu_resume_after_removals(tmp_path):
    """Resume on the GPU from a state file written after particles left a
    hopper through the bottom of the box: its records whose partners lie past
    the last particle come back as they were, and the run stays
    bit-identical with the uninterrupted GPU run and the oracle."""
    w = configs.discharge(d_out=5.0, mu=0.2)

    def fresh(make):
        s = make(w.params)
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        return s

    full = fresh(DEMSystem)
    full.run(1, 700)
    part = fresh(DEMSystem)
    part.run(1, 450)
    comps = SF.component_records([P.Component(part.n, 1.0, configs.DENSITY, 2.0 * configs.KN,
                                              2.0 * configs.KT)])
    st = SF.capture(part, components=comps, wall_stiffness=[(1.0, 1.0)], step=450)
    assert np.any(st.contacts["imax"] >= part.n)
    path = os.path.join(tmp_path, "d.stt")
    SF.write_state(path, st)
    back = SF.read_state(path, w.params.method_order - 1)
    res = DEMSystem(SF.params_with_walls(w.params, back))
    res.run(SF.restore(res, back), 700)
    _same(full, res, "gpu resume after removals")
    o = fresh(oracle_system)
    o.run(1, 700)
    _same(full, o, "gpu vs oracle")


def test_gpu_resume_while_pouring(tmp_path):
    """The shipped example (pouring, orbiting cone walls) saved on the GPU
    mid-pour and resumed on the GPU: bit-identical with the uninterrupted
    GPU run, which is bit-identical with the oracle's."""
    from tests.test_ball_bearings import start
    from tests.test_particle_removal import export
    from tests.test_statefile import _resume_ball_bearings
    full = _resume_ball_bearings(DEMSystem, tmp_path)
    _, _, _, o = start(oracle_system)
    o.run(1, 24000)
    a, b = export(full, True), export(o, True)
    for k in ("pos", "vel", "cell_index", "traversal", "cell_start", "prev"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert full.rng() == o.rng()
