"""State files in the reference's layout (SaveState/ReadState,
src/DEM.f90:947-1134): byte layout, round trip, and a resumed oracle run that
is bit-identical with the uninterrupted one."""
import os

import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200 import statefile as SF
from tests.oracle_lib import oracle_system


def _random_state(rng, n=37, nc=2, nw=2, nprev=3, ncell=11):
    comps = []
    index = rng.integers(0, nc, n).astype(np.int32)
    for k in range(nc):
        comps.append(SF.ComponentRecord(int(np.count_nonzero(index == k)), *rng.random(6)))
    walls = [SF.WallRecord(1 + (j % 2), *rng.random(3), *rng.random((6, 3)), *rng.random(2))
             for j in range(nw)]
    cfg = SF.Configuration(1.5, 2.5, 3.5, 0.125, rng.random(3), comps, walls, index,
                           rng.random((n, 3)), rng.random((n, 3)), rng.random((n, 3)))
    cut = np.sort(rng.integers(0, n + 1, ncell - 1))
    cell_start = np.concatenate([[0], cut, [n]]).astype(np.int32)
    trav = rng.permutation(n).astype(np.int32)
    m, mw = 25, 9
    imin = np.sort(rng.integers(0, n - 1, m)).astype(np.int32)
    ip = np.sort(rng.integers(0, n, mw)).astype(np.int32)
    ct = dict(imin=imin, imax=(imin + 1).astype(np.int32), ft=rng.random((m, 3)),
              vt=rng.random((m, 3)), ip=ip, iw=rng.integers(0, nw, mw).astype(np.int32),
              ftw=rng.random((mw, 3)), vtw=rng.random((mw, 3)))
    return SF.StateFile(cfg, trav, cell_start, np.array([2, 3, 1], np.int32)[:nprev],
                        rng.random((nprev, n, 9)), ct, 1234, 98765, False,
                        "Jan 1st 2026 at 10:00:00", [("a", "b")], "Jan 2nd 2026 at 11:00:00",
                        (5, 6, 7, 890), (0.5, 3, 4, 5, 6), 17)


def test_state_file_round_trip_and_layout(tmp_path):
    rng = np.random.default_rng(5)
    s = _random_state(rng)
    path = os.path.join(tmp_path, "x.stt")
    SF.write_state(path, s)
    n, nc, nw, nprev, ncell = 37, 2, 2, 3, 11
    m, mw = 25, 9
    header = 2 + 28 + 4 + 2 * 28 + 28 + (4 + 1 + 1 + 2)
    cfg = (4 + 3 + 8 * 4 + 24 + 4 + nc * (4 + 6 * 8) + 4 + nw * (4 + 3 * 8 + 6 * 24 + 16) + 1
           + n * (4 + 9 * 8))
    cells = 4 + 4 * ncell + 4 * n
    integ = 4 * nprev + nprev * n * 72
    contacts = 4 + n * 8 + (m + mw) * (4 + 48)
    tail = 8 + 4 * 4 + 4 + 4 + 4
    data = open(path, "rb").read()
    assert len(data) == header + cfg + cells + integ + contacts + tail
    assert data[header:header + 4] == b"DEMC"
    assert data[header + 4:header + 7] == bytes([2, 3, 72])
    r = SF.read_state(path, nprev)
    assert r.initial_step == 1234 and r.ncol == 98765 and r.conf == 17
    assert r.start_time == s.start_time and r.interruptions == s.interruptions
    assert r.duration == s.duration and r.rng == s.rng
    for a in ("pos", "vel", "omega", "index", "lbox"):
        np.testing.assert_array_equal(getattr(r.config, a), getattr(s.config, a))
    assert r.config.components == s.config.components
    for a, b in zip(r.config.walls, s.config.walls):
        for k in ("shape", "l1", "l2", "l3", "stiffness", "shear_stiffness"):
            assert getattr(a, k) == getattr(b, k)
        for k in ("u", "w", "n", "position", "velocity", "omega"):
            np.testing.assert_array_equal(getattr(a, k), getattr(b, k))
    np.testing.assert_array_equal(r.traversal, s.traversal)
    np.testing.assert_array_equal(r.cell_start, s.cell_start)
    np.testing.assert_array_equal(r.ipc, s.ipc)
    np.testing.assert_array_equal(r.previous, s.previous)
    for k in s.contacts:
        np.testing.assert_array_equal(r.contacts[k], s.contacts[k], err_msg=k)
    # a truncated file is an error, as BinFiles' "end of file exceeded"
    with open(path, "wb") as f:
        f.write(data[:-3])
    with pytest.raises(ValueError):
        SF.read_state(path, nprev)


def test_configuration_file_round_trip(tmp_path):
    s = _random_state(np.random.default_rng(6))
    path = os.path.join(tmp_path, "x.cfg")
    SF.write_configuration(path, s.config)
    c = SF.read_configuration(path)
    np.testing.assert_array_equal(c.pos, s.config.pos)
    assert c.time == s.config.time and c.components == s.config.components


def _hopper_pair(w, motion):
    sys = oracle_system(w.params)
    sys.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
    sys.initialize_cell_distribution()
    if motion:
        sys.set_wall_motion(motion)
    return sys


def _vibration(w):
    cone, floor = w.params.walls[0], w.params.walls[1]
    return [P.wall_motion(list(cone.position), (0.0, 0.0, 0.03), (0.0, 0.0, 25.0),
                          (0.0, 0.0, 0.6)),
            P.wall_motion(list(floor.position), (0.0, 0.0, 0.02), (0.0, 0.0, 20.0),
                          (0.0, 0.0, 0.1))]


@pytest.mark.parametrize("moving", [False, True])
def test_oracle_resume_is_bit_identical(tmp_path, moving):
    """Save after step k, read back into a fresh context, run on: the same
    bits as the uninterrupted run (cell lists, ring, contacts, Ncol restored)."""
    w = configs.hopper(n=300, seed=1011, euler_intervals=8)
    motion = _vibration(w) if moving else None
    full = _hopper_pair(w, motion)
    full.run(1, 260)
    part = _hopper_pair(w, motion)
    part.run(1, 150)
    comps = SF.component_records([P.Component(300, 1.0, configs.DENSITY, 2.0 * configs.KN,
                                              2.0 * configs.KT)])
    state = SF.capture(part, components=comps, wall_stiffness=[(1.0, 2.0), (3.0, 4.0)],
                       step=150, start_time="Dec 3rd 2026 at 12:00:00")
    path = os.path.join(tmp_path, "hopper.stt")
    SF.write_state(path, state)
    back = SF.read_state(path, w.params.method_order - 1)
    assert back.initial_step == 151 and back.ncol == part.ncol()
    res = oracle_system(SF.params_with_walls(w.params, back))
    if motion:
        res.set_wall_motion(motion)
    first = SF.restore(res, back)
    res.run(first, 260)
    a, b = full.get_state(), res.get_state()
    for k in ("pos", "vel", "omega"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    ca, cb = full.get_contacts(), res.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    for x, y in zip(full.get_cells(), res.get_cells()):
        np.testing.assert_array_equal(x, y)
    assert full.ncol() == res.ncol()
    np.testing.assert_array_equal(full.walls()["position"], res.walls()["position"])


def test_set_cells_rejects_inconsistent_lists():
    w = configs.hopper(n=50, seed=1012)
    o = _hopper_pair(w, None)
    _, tr, cs = o.get_cells()
    bad = tr.copy()
    bad[[0, -1]] = bad[[-1, 0]]  # two particles in each other's cells
    from dem3d_b200.system import DEMError
    if not np.array_equal(o.get_cells()[0][tr[0]], o.get_cells()[0][tr[-1]]):
        with pytest.raises(DEMError):
            o.set_cells(bad, cs)
    dup = tr.copy()
    dup[1] = dup[0]
    with pytest.raises(DEMError):
        o.set_cells(dup, cs)
    o.set_cells(tr, cs)  # the lists as they are: accepted


def test_oracle_resume_after_removals(tmp_path):
    """A hopper emptying through the bottom of the box: the state file is
    written after particles have left (records with partners past the last
    particle included), and the resumed run stays bit-identical."""
    w = configs.discharge(d_out=5.0, mu=0.2)

    def fresh():
        s = oracle_system(w.params)
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        return s

    full = fresh()
    full.run(1, 700)
    part = fresh()
    part.run(1, 450)
    assert part.n < w.pos.shape[0]  # some particles have left
    comps = SF.component_records([P.Component(part.n, 1.0, configs.DENSITY, 2.0 * configs.KN,
                                              2.0 * configs.KT)])
    st = SF.capture(part, components=comps, wall_stiffness=[(1.0, 1.0)], step=450)
    path = os.path.join(tmp_path, "d.stt")
    SF.write_state(path, st)
    back = SF.read_state(path, w.params.method_order - 1)
    res = oracle_system(SF.params_with_walls(w.params, back))
    res.run(SF.restore(res, back), 700)
    a, b = full.get_state(), res.get_state()
    assert full.n == res.n
    for k in ("pos", "vel", "omega"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    ca, cb = full.get_contacts(), res.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    assert full.ncol() == res.ncol()
