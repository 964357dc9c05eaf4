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


class _Fread:
    """MATLAB's fread(file, count, precision) on a little-endian byte string."""

    def __init__(self, data):
        self.data, self.at = data, 0

    def __call__(self, count, fmt):
        size = {"int8": 1, "int32": 4, "float64": 8}[fmt]
        code = {"int8": "<i1", "int32": "<i4", "float64": "<f8"}[fmt]
        out = np.frombuffer(self.data, dtype=code, count=count, offset=self.at)
        self.at += count * size
        return out.astype(np.float64)


def _matlab_readfile(data):
    """The Complete branch of the reference's MATLAB reader, matlab/readfile.m,
    in its order of fread calls (ib = int32, rb = float64, dim = 3)."""
    fread = _Fread(data)
    out = {}
    assert fread(1, "int32")[0] == 1129137476                       # :25-26
    version = int(fread(1, "int8")[0])                               # :27
    dim = int(fread(1, "int8")[0])
    dav, ini = 2 * dim - 3, 7 - 2 * dim                              # :29-30
    full = int(fread(1, "int8")[0]) == 72                            # :31-33
    assert full and dim == 3
    out["scales"] = [fread(1, "float64")[0] for _ in range(3)]      # :35-37
    out["time"] = fread(1, "float64")[0]                             # :38
    out["lbox"] = fread(dim, "float64")                              # :39
    comps = []
    for _ in range(int(fread(1, "int32")[0])):                       # :43-66
        rec = [fread(1, "int32")[0], fread(1, "float64")[0], fread(1, "float64")[0],
               fread(1, "float64")[0]]
        rec.append(fread(1, "float64")[0] if version == 2 else 2.0 / 7.0 * rec[3])
        rec += [fread(1, "float64")[0], fread(1, "float64")[0]]
        comps.append(rec)
    out["components"] = comps
    walls = []
    for _ in range(int(fread(1, "int32")[0])):                       # :69-112
        wl = {"type": fread(1, "int32")[0], "l": fread(3, "float64")}
        for k in ("u", "w", "n", "position", "velocity"):
            wl[k] = fread(dim, "float64")
        om = np.zeros(3)
        om[ini - 1:] = fread(dav, "float64")
        wl["omega"] = om
        if version == 2:
            wl["k"] = (fread(1, "float64")[0], fread(1, "float64")[0])
        walls.append(wl)
    out["walls"] = walls
    vectors = fread(1, "int8")[0] != 0                               # :115
    npart = int(sum(c[0] for c in comps))                            # :114
    idx, x, v, w = [], [], [], []
    for _ in range(npart):                                           # :131-141
        idx.append(fread(1, "int32")[0])
        x.append(fread(dim, "float64"))
        v.append(fread(dim, "float64"))
        w.append(fread(dav, "float64"))
        if vectors:
            fread(3 * dim, "float64")
    out.update(index=np.array(idx), pos=np.array(x), vel=np.array(v), omega=np.array(w))
    out["consumed"] = fread.at
    return out


def test_configuration_reads_with_the_matlab_reader(tmp_path):
    """The Complete configuration written here is what the reference's own
    MATLAB reader expects, field by field, to the last byte."""
    rng = np.random.default_rng(8)
    cfg = _random_state(rng, n=23, nc=3, nw=3).config
    path = os.path.join(tmp_path, "x.cfg")
    SF.write_configuration(path, cfg)
    data = open(path, "rb").read()
    m = _matlab_readfile(data)
    assert m["consumed"] == len(data)
    assert m["scales"] == [cfg.length_scale, cfg.time_scale, cfg.mass_scale]
    assert m["time"] == cfg.time
    np.testing.assert_array_equal(m["lbox"], cfg.lbox)
    for got, k in zip(m["components"], cfg.components):
        assert got == [k.number, k.radius, k.density, k.stiffness, k.shear_stiffness, k.mass,
                       k.inertia]
    for got, wl in zip(m["walls"], cfg.walls):
        assert got["type"] == wl.shape
        np.testing.assert_array_equal(got["l"], [wl.l1, wl.l2, wl.l3])
        for k in ("u", "w", "n", "position", "velocity", "omega"):
            np.testing.assert_array_equal(got[k], getattr(wl, k))
        assert got["k"] == (wl.stiffness, wl.shear_stiffness)
    np.testing.assert_array_equal(m["index"], cfg.index + 1)
    for k in ("pos", "vel", "omega"):
        np.testing.assert_array_equal(m[k], getattr(cfg, k))


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


def _resume_ball_bearings(make, tmp_path, save_at=12000, end=24000):
    """The shipped example saved mid-pour and resumed: the generator, the
    poured spheres, the orbiting cones and the contacts come back, and the
    resumed run continues as the uninterrupted one."""
    from tests.test_ball_bearings import start
    from tests.test_particle_removal import export
    w, motion, pour, full = start(make)
    full.run(1, end)
    _, _, _, part = start(make)
    part.run(1, save_at)
    assert 0 < part.n < full.n
    comps = SF.component_records([P.Component(part.n, 1.0, configs.DENSITY, 2.0 * configs.KN,
                                              2.0 * configs.KT)])
    st = SF.capture(part, components=comps, wall_stiffness=[(1.0, 1.0)] * 5, step=save_at)
    path = os.path.join(tmp_path, "bb.stt")
    SF.write_state(path, st)
    back = SF.read_state(path, w.params.method_order - 1)
    res = make(SF.params_with_walls(w.params, back))
    res.set_wall_motion(motion)
    res.set_pouring(pour)
    assert SF.restore(res, back) == save_at + 1
    assert res.rng() == part.rng()
    res.run(save_at + 1, end)
    a, b = export(full, True), export(res, True)
    for k in ("pos", "vel", "cell_index", "traversal", "cell_start", "prev"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in a["contacts"]:
        np.testing.assert_array_equal(a["contacts"][k], b["contacts"][k], err_msg=k)
    assert full.rng() == res.rng() and full.ncol() == res.ncol()
    np.testing.assert_array_equal(full.walls()["position"], res.walls()["position"])
    return full


def test_oracle_resume_while_pouring(tmp_path):
    _resume_ball_bearings(oracle_system, tmp_path)


def test_double_buffered_saves_and_resume_choice(tmp_path):
    """SaveState alternates between the two state files and a resumed run
    reads the first one that exists, whatever their ages."""
    a, b = os.path.join(tmp_path, "r.stt"), os.path.join(tmp_path, "r.st2")
    picks = [SF.state_file_for_step(k, 100, a, b) for k in range(50, 650, 50)]
    assert picks == [None, a, None, b, None, a, None, b, None, a, None, b]
    assert SF.state_file_for_step(123, 100, a, b, finished=True) == b
    assert SF.resume_file(a, b) is None
    open(b, "wb").close()
    assert SF.resume_file(a, b) == b
    open(a, "wb").close()
    assert SF.resume_file(a, b) == a


def test_periodic_saves_and_resume_after_a_crash(tmp_path):
    """A run that saves every 60 steps into the two files stops at step 250
    (as if it had crashed). The resumed run reads the first file that exists,
    the one written at step 180 (the other one holds step 240), and reaches
    step 400 bit-identical with the uninterrupted run."""
    w = configs.hopper(n=300, seed=1006)
    comps = SF.component_records([P.Component(len(w.pos), 1.0, configs.DENSITY,
                                              2.0 * configs.KN, 2.0 * configs.KT)])
    stiff = [(2.0 * configs.KN, 2.0 * configs.KT)] * w.params.n_walls
    a, b = os.path.join(tmp_path, "h.stt"), os.path.join(tmp_path, "h.st2")

    def fresh(params):
        s = oracle_system(params)
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        return s
    full = fresh(w.params)
    full.run(1, 400)
    crashed = fresh(w.params)
    for first, last in ((1, 60), (61, 120), (121, 180), (181, 240), (241, 250)):
        crashed.run(first, last)
        path = SF.state_file_for_step(last, 60, a, b)
        if path:
            SF.write_state(path, SF.capture(crashed, components=comps, wall_stiffness=stiff,
                                            step=last))
    path = SF.resume_file(a, b)
    assert path == a
    back = SF.read_state(path, w.params.method_order - 1)
    assert back.initial_step == 181
    res = oracle_system(SF.params_with_walls(w.params, back))
    res.run(SF.restore(res, back), 400)
    sa, sb = full.get_state(), res.get_state()
    for k in ("pos", "vel", "omega"):
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    ca, cb = full.get_contacts(), res.get_contacts()
    for k in ca:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    assert full.ncol() == res.ncol()


def test_corrupt_state_files_are_errors(tmp_path):
    """A file that is not a state file, or holds another dimension, is an
    error, as ReadConfFromUnit's checks are (src/MConfig.f90:109-448)."""
    rng = np.random.default_rng(9)
    path = os.path.join(tmp_path, "c.stt")
    SF.write_state(path, _random_state(rng))
    data = bytearray(open(path, "rb").read())
    at = data.index(b"DEMC")
    for offset, value in ((0, ord("X")), (5, 2)):   # signature; int(dim,1)
        bad = bytearray(data)
        bad[at + offset] = value
        with open(path, "wb") as f:
            f.write(bad)
        with pytest.raises(ValueError):
            SF.read_state(path, 3)
