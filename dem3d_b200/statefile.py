"""The reference's state file (``.stt``) and Complete configuration (``.cfg``).

A state file lets a run stop and resume, on the CUDA library or on the
Fortran program, from the same bytes.  The layout restates the writers and
readers of the reference:

* ``SaveState`` / ``ReadState`` (src/DEM.f90:947-1014, 1018-1134): header,
  configuration, cell lists, integration ring, contact lists, generator state,
  configuration index, next step, Ncol;
* ``SaveConfToUnit`` / ``ReadConfFromUnit`` in the Complete form
  (src/MConfig.f90:109-243, 265-448);
* ``SaveCellStructure`` / ``ReadCellStructure`` (src/MCells.f90:958-1026);
* ``Save/ReadIntegrationVariables`` (src/MDEM.f90:52-89);
* ``Save/ReadContactList`` (src/MContacts.f90:75-169).

``BinFiles`` (src/BinFiles.f90) writes each value's bytes back to back, with
no record markers, and flushes the last partial buffer in halving slices, so
a file is exactly the concatenation of its values: ``integer(ib)`` as int32,
``real(rb)`` as float64, ``logical(lb)`` as 2 bytes, ``logical(1)`` and
``integer(1)`` as 1 byte, strings as their fixed length, all little-endian
(the byte order of the machines the reference runs on).

All quantities are in simulation units (after ``ScaleVariables``), as the
reference stores them.  Indices are 1-based in the file and 0-based here.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

FOURCC = b"DEMC"          # src/MConfig.f90:11
CFG_VERSION = 2           # src/MConfig.f90:14
COMPLETE = 72             # src/MConfig.f90:20
COMPACT = 28
STR_LEN = 28              # character(28) of StrDateAndTime (src/MTime.f90:199)


@dataclass
class ComponentRecord:
    """TComponent fields that a Complete configuration holds."""

    number: int
    radius: float
    density: float
    stiffness: float
    shear_stiffness: float
    mass: float
    inertia: float


@dataclass
class WallRecord:
    """TWall (src/MDimension3D.f90:45-59) as a Complete configuration holds it
    (``Order`` is not stored: ConfigureWalls derives it)."""

    shape: int
    l1: float
    l2: float
    l3: float
    u: np.ndarray
    w: np.ndarray
    n: np.ndarray
    position: np.ndarray
    velocity: np.ndarray
    omega: np.ndarray
    stiffness: float
    shear_stiffness: float


@dataclass
class Configuration:
    length_scale: float
    time_scale: float
    mass_scale: float
    time: float
    lbox: np.ndarray
    components: list
    walls: list
    index: np.ndarray       # Particle%Index - 1 (component, 0-based)
    pos: np.ndarray
    vel: np.ndarray
    omega: np.ndarray
    directions: tuple | None = None   # (U, W, N), each (n, 3), when stored
    version: int = CFG_VERSION


@dataclass
class StateFile:
    config: Configuration
    traversal: np.ndarray        # cell lists, particles in list order (0-based)
    cell_start: np.ndarray       # Nt + 1 offsets into traversal
    ipc: np.ndarray              # ipc(1:NPrev), 1-based physical slots
    previous: np.ndarray         # (NPrev, n, 9): v, a, alpha per physical slot
    contacts: dict               # imin, imax, ft, vt, ip, iw, ftw, vtw (0-based)
    initial_step: int            # the step a resumed run starts with
    ncol: int
    finished: bool = False
    start_time: str = ""
    interruptions: list = field(default_factory=list)  # (interrupted, retaken) pairs
    finish_time: str = ""
    duration: tuple = (0, 0, 0, 0)  # hours, minutes, seconds, milliseconds
    rng: tuple = (0.0, 0, -1, -1, 0)  # aam, Dummy, iix, iiy, iik (src/MUtil.f90:10-11)
    conf: int = 0
    n_main: int | None = None    # size(MainParticle) when larger than NP


# ---------------------------------------------------------------------------
# byte stream


class _Writer:
    def __init__(self):
        self.parts = []

    def i1(self, v):
        self.parts.append(struct.pack("<b", int(v)))

    def i2(self, v):
        self.parts.append(struct.pack("<h", int(v)))

    def i4(self, v):
        self.parts.append(struct.pack("<i", int(v)))

    def f8(self, v):
        self.parts.append(struct.pack("<d", float(v)))

    def l1(self, v):
        self.parts.append(b"\x01" if v else b"\x00")

    def l2(self, v):
        self.parts.append(struct.pack("<h", 1 if v else 0))

    def s(self, text, n=STR_LEN):
        b = text.encode("ascii")[:n]
        self.parts.append(b + b" " * (n - len(b)))

    def raw(self, b):
        self.parts.append(bytes(b))

    def vec(self, a):
        self.parts.append(np.ascontiguousarray(a, dtype="<f8").tobytes())

    def ivec(self, a):
        self.parts.append(np.ascontiguousarray(a, dtype="<i4").tobytes())

    def bytes(self):
        return b"".join(self.parts)


class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        self.p = 0

    def _take(self, n):
        if self.p + n > len(self.d):
            raise ValueError("end of file exceeded")  # BinFiles error 7
        b = self.d[self.p:self.p + n]
        self.p += n
        return b

    def i1(self):
        return struct.unpack("<b", self._take(1))[0]

    def i2(self):
        return struct.unpack("<h", self._take(2))[0]

    def i4(self):
        return struct.unpack("<i", self._take(4))[0]

    def f8(self):
        return struct.unpack("<d", self._take(8))[0]

    def l1(self):
        return self._take(1) != b"\x00"

    def l2(self):
        return self._take(2) != b"\x00\x00"

    def s(self, n=STR_LEN):
        return self._take(n).decode("ascii", "replace").rstrip(" ")

    def vec(self, count):
        return np.frombuffer(self._take(8 * count), dtype="<f8").astype(np.float64)

    def ivec(self, count):
        return np.frombuffer(self._take(4 * count), dtype="<i4").astype(np.int32)


# ---------------------------------------------------------------------------
# configuration (SaveConfToUnit / ReadConfFromUnit, Complete form)


def _put_configuration(w: _Writer, c: Configuration) -> None:
    n = len(c.pos)
    w.raw(FOURCC)
    w.i1(c.version)
    w.i1(3)          # int(dim,1)
    w.i1(COMPLETE)
    w.f8(c.length_scale)
    w.f8(c.time_scale)
    w.f8(c.mass_scale)
    w.f8(c.time)
    w.vec(c.lbox)
    w.i4(len(c.components))
    for k in c.components:
        w.i4(k.number)
        w.f8(k.radius)
        w.f8(k.density)
        w.f8(k.stiffness)
        w.f8(k.shear_stiffness)
        w.f8(k.mass)
        w.f8(k.inertia)
    w.i4(len(c.walls))
    for x in c.walls:
        w.i4(x.shape)
        w.f8(x.l1)
        w.f8(x.l2)
        w.f8(x.l3)
        w.vec(x.u)
        w.vec(x.w)
        w.vec(x.n)
        w.vec(x.position)
        w.vec(x.velocity)
        w.vec(x.omega)   # WriteAxialVector (src/MDimension3D.f90:99-107)
        w.f8(x.stiffness)
        w.f8(x.shear_stiffness)
    w.l1(c.directions is not None)
    counts = np.bincount(np.asarray(c.index), minlength=len(c.components))
    if len(counts) != len(c.components) or any(
            int(counts[i]) != int(k.number) for i, k in enumerate(c.components)):
        raise ValueError("Component%Number must count the particles of each component")
    rec = np.empty((n, 3 if c.directions is None else 6, 3))
    rec[:, 0] = c.pos
    rec[:, 1] = c.vel
    rec[:, 2] = c.omega
    if c.directions is not None:
        for k in range(3):
            rec[:, 3 + k] = c.directions[k]
    # each particle: Index (int32) then its vectors, back to back
    body = np.empty(n, dtype=[("index", "<i4"), ("v", "<f8", (rec.shape[1] * 3,))])
    body["index"] = np.asarray(c.index, dtype=np.int32) + 1
    body["v"] = rec.reshape(n, -1)
    w.raw(body.tobytes())


def _get_configuration(r: _Reader) -> Configuration:
    if r._take(4) != FOURCC:
        raise ValueError("not a configuration file")
    version = r.i1()
    if r.i1() != 3:
        raise ValueError("invalid dimension")
    form = r.i1()
    full = form == COMPLETE
    length_scale = r.f8()
    time_scale = r.f8()
    mass_scale = r.f8() if full else 1.0
    time = r.f8()
    lbox = r.vec(3)
    nc = r.i4()
    comps = []
    for _ in range(nc):
        number = r.i4()
        radius = r.f8()
        if full:
            density = r.f8()
            stiff = r.f8()
            shear = r.f8() if version == 2 else 2.0 / 7.0 * stiff
            comps.append(ComponentRecord(number, radius, density, stiff, shear, r.f8(), r.f8()))
        else:
            comps.append(ComponentRecord(number, radius, 0.0, 0.0, 0.0, 0.0, 0.0))
    nw = r.i4()
    walls = []
    for _ in range(nw):
        shape = r.i4()
        l1, l2, l3 = r.f8(), r.f8(), r.f8()
        if not full:
            raise ValueError("Compact configurations are snapshots; a state file holds a "
                             "Complete one")
        u, w_, n_ = r.vec(3), r.vec(3), r.vec(3)
        pos = r.vec(3)
        vel, om = r.vec(3), r.vec(3)
        ks, kt = (r.f8(), r.f8()) if version == 2 else (0.0, 0.0)
        walls.append(WallRecord(shape, l1, l2, l3, u, w_, n_, pos, vel, om, ks, kt))
    n = int(sum(k.number for k in comps))
    vectors = r.l1()
    if not full:
        raise ValueError("Compact configurations are not read here")
    nv = 6 if vectors else 3
    body = np.frombuffer(r._take(n * (4 + 8 * 3 * nv)),
                         dtype=[("index", "<i4"), ("v", "<f8", (nv * 3,))])
    v = body["v"].astype(np.float64).reshape(n, nv, 3)
    dirs = (v[:, 3].copy(), v[:, 4].copy(), v[:, 5].copy()) if vectors else None
    return Configuration(length_scale, time_scale, mass_scale, time, lbox, comps, walls,
                         body["index"].astype(np.int32) - 1, v[:, 0].copy(), v[:, 1].copy(),
                         v[:, 2].copy(), dirs, version)


def write_configuration(path: str, c: Configuration) -> None:
    """SaveConfToFile(File, Complete) (src/MConfig.f90:88-103)."""
    w = _Writer()
    _put_configuration(w, c)
    with open(path, "wb") as f:
        f.write(w.bytes())


def read_configuration(path: str) -> Configuration:
    with open(path, "rb") as f:
        return _get_configuration(_Reader(f.read()))


# ---------------------------------------------------------------------------
# state file


def write_state(path: str, s: StateFile) -> None:
    """SaveState (src/DEM.f90:947-1014)."""
    c = s.config
    n = len(c.pos)
    w = _Writer()
    w.l2(s.finished)
    w.s(s.start_time)
    w.i4(len(s.interruptions))
    for a, b in s.interruptions:
        w.s(a)
        w.s(b)
    w.s(s.finish_time)
    h, m, sec, ms = s.duration
    w.i4(h)
    w.i1(m)
    w.i1(sec)
    w.i2(ms)
    _put_configuration(w, c)
    # SaveCellStructure: Nt, then per cell its count and particle indices
    cs = np.asarray(s.cell_start, dtype=np.int64)
    tr = np.asarray(s.traversal, dtype=np.int32)
    nt = len(cs) - 1
    if cs[0] != 0 or cs[-1] != n or len(tr) != n:
        raise ValueError("cell lists must hold every particle")
    counts = np.diff(cs).astype(np.int32)
    out = np.empty(nt + n, dtype="<i4")
    # the count of cell k sits before its members: offsets shifted by k + 1
    pos_count = cs[:-1] + np.arange(nt)
    out[pos_count] = counts
    member_pos = np.arange(n) + np.repeat(np.arange(nt) + 1, counts)
    out[member_pos] = tr + 1
    w.i4(nt)
    w.raw(out.tobytes())
    # SaveIntegrationVariables: ipc(1:NPrev), then Previous(j,i) j-major
    ipc = np.asarray(s.ipc, dtype=np.int32)
    w.ivec(ipc)
    prev = np.asarray(s.previous, dtype=np.float64).reshape(len(ipc), n, 9)
    w.vec(prev)
    # SaveContactList: for each main particle its partner list then its wall list
    _put_contacts(w, s.contacts, s.n_main if s.n_main is not None else n)
    aam, dummy, iix, iiy, iik = s.rng
    w.f8(aam)
    w.i4(dummy)
    w.i4(iix)
    w.i4(iiy)
    w.i4(iik)
    w.i4(s.conf)
    w.i4(s.initial_step)
    w.i4(np.int64(s.ncol).astype(np.int32))  # integer(ib) Ncol
    with open(path, "wb") as f:
        f.write(w.bytes())


def _put_contacts(w: _Writer, ct: dict, n_main: int) -> None:
    rec = np.dtype([("index", "<i4"), ("v1", "<f8", (3,)), ("v2", "<f8", (3,))])
    imin = np.asarray(ct["imin"], dtype=np.int64)
    ip = np.asarray(ct["ip"], dtype=np.int64)
    pp = np.zeros(len(imin), dtype=rec)
    pp["index"] = np.asarray(ct["imax"]) + 1
    pp["v1"] = ct["ft"]
    pp["v2"] = ct["vt"]
    pw = np.zeros(len(ip), dtype=rec)
    pw["index"] = np.asarray(ct["iw"]) + 1
    pw["v1"] = ct["ftw"]
    pw["v2"] = ct["vtw"]
    # the lists are grouped by main particle (records come sorted by it)
    if np.any(np.diff(imin) < 0) or np.any(np.diff(ip) < 0):
        raise ValueError("contact records must be grouped by main particle")
    a = np.searchsorted(imin, np.arange(n_main + 1))
    b = np.searchsorted(ip, np.arange(n_main + 1))
    w.i4(n_main)
    for i in range(n_main):
        w.i4(a[i + 1] - a[i])
        w.raw(pp[a[i]:a[i + 1]].tobytes())
        w.i4(b[i + 1] - b[i])
        w.raw(pw[b[i]:b[i + 1]].tobytes())


def _get_contacts(r: _Reader):
    rec = np.dtype([("index", "<i4"), ("v1", "<f8", (3,)), ("v2", "<f8", (3,))])
    n_main = r.i4()
    pairs, walls, owner_p, owner_w = [], [], [], []
    for i in range(n_main):
        k = r.i4()
        if k:
            pairs.append(np.frombuffer(r._take(k * rec.itemsize), dtype=rec))
            owner_p.append(np.full(k, i, dtype=np.int32))
        k = r.i4()
        if k:
            walls.append(np.frombuffer(r._take(k * rec.itemsize), dtype=rec))
            owner_w.append(np.full(k, i, dtype=np.int32))
    pp = np.concatenate(pairs) if pairs else np.zeros(0, dtype=rec)
    pw = np.concatenate(walls) if walls else np.zeros(0, dtype=rec)
    ct = dict(imin=np.concatenate(owner_p) if owner_p else np.zeros(0, np.int32),
              imax=pp["index"].astype(np.int32) - 1, ft=pp["v1"].astype(np.float64),
              vt=pp["v2"].astype(np.float64),
              ip=np.concatenate(owner_w) if owner_w else np.zeros(0, np.int32),
              iw=pw["index"].astype(np.int32) - 1, ftw=pw["v1"].astype(np.float64),
              vtw=pw["v2"].astype(np.float64))
    return ct, n_main


def state_file_for_step(step: int, save_interval: int, state_file: str, state_file2: str,
                        finished: bool = False):
    """The file PerformPeriodicTasks saves after ``step`` (src/DEM.f90:164-170),
    or None: every ``save_interval`` steps, alternately ``state_file`` and
    ``state_file2`` (the second one on multiples of twice the interval and when
    the run has finished), so that a crash while writing one leaves the
    other intact."""
    if step % save_interval != 0 and not finished:
        return None
    return state_file2 if (step % (2 * save_interval) == 0 or finished) else state_file


def resume_file(state_file: str, state_file2: str):
    """The file a resumed run reads (src/DEM.f90:73-83): ``state_file`` if it
    exists, else ``state_file2``, else None (the run starts afresh).  As in
    the reference, the two files' ages are not compared."""
    import os
    for path in (state_file, state_file2):
        if os.path.exists(path):
            return path
    return None


def read_state(path: str, nprev: int) -> StateFile:
    """ReadState (src/DEM.f90:1018-1134).  ``nprev`` = MethodOrder - 1 comes
    from the specification, as in the reference (the file does not hold it)."""
    with open(path, "rb") as f:
        r = _Reader(f.read())
    finished = r.l2()
    start = r.s()
    ni = r.i4()
    inter = [(r.s(), r.s()) for _ in range(ni)]
    finish = r.s()
    duration = (r.i4(), r.i1(), r.i1(), r.i2())
    cfg = _get_configuration(r)
    n = len(cfg.pos)
    nt = r.i4()
    cell_start = np.zeros(nt + 1, dtype=np.int32)
    trav = np.empty(n, dtype=np.int32)
    k = 0
    for cc in range(nt):
        m = r.i4()
        if k + m > n:
            raise ValueError("cell lists hold more particles than the configuration")
        trav[k:k + m] = r.ivec(m) - 1
        k += m
        cell_start[cc + 1] = k
    if k != n:
        raise ValueError("cell lists do not hold every particle")
    ipc = r.ivec(nprev)
    prev = r.vec(nprev * n * 9).reshape(nprev, n, 9)
    ct, n_main = _get_contacts(r)
    rng = (r.f8(), r.i4(), r.i4(), r.i4(), r.i4())
    conf = r.i4()
    step = r.i4()
    ncol = r.i4()
    if r.p != len(r.d):
        raise ValueError("trailing bytes after Ncol")
    return StateFile(cfg, trav, cell_start, ipc, prev, ct, step, ncol, finished, start, inter,
                     finish, duration, rng, conf, n_main if n_main != n else None)


# ---------------------------------------------------------------------------
# a running system <-> a state file


def component_records(components, scales=None) -> list:
    """Component(:) as the reference holds it after CalculateProperties and
    ScaleVariables (src/DEM.f90:807-833): radius, mass and inertia derived
    from the diameter and density, all in simulation units when ``scales``
    (a :class:`~dem3d_b200.params.Scales`) is given."""
    from .params import PI
    out = []
    for k in components:
        r = 0.5 * k.diameter
        m = 4.0 * PI / 3.0 * (r * r * r) * k.density
        i = 2.0 / 5.0 * m * (r * r)
        rec = ComponentRecord(k.number, r, k.density, k.stiffness, k.shear_stiffness, m, i)
        if scales is not None:
            L, M, T = scales.length, scales.mass, scales.time
            rec = ComponentRecord(k.number, r / L, k.density * L ** 3 / M,
                                  k.stiffness * T ** 2 / M, k.shear_stiffness * T ** 2 / M,
                                  m / M, i / (L ** 2 * M))
        out.append(rec)
    return out


def wall_stiffness(walls, scales=None) -> list:
    """(Wall%Stiffness, Wall%ShearStiffness) per wall, scaled like
    ScaleVariables when ``scales`` is given."""
    f = 1.0 if scales is None else scales.time ** 2 / scales.mass
    return [(w.stiffness * f, w.shear_stiffness * f) for w in walls]


def capture(system, *, components, wall_stiffness, step: int, scales=(1.0, 1.0, 1.0),
            comp=None, **header) -> StateFile:
    """What SaveState would write after ``step`` of ``system`` (a
    :class:`~dem3d_b200.system.DEMSystem`).

    ``components``: a :class:`ComponentRecord` per component (scaled values;
    ``number`` is recounted); ``wall_stiffness``: (Stiffness, ShearStiffness)
    per wall; ``scales``: (LengthScale, TimeScale, MassScale); ``comp``: the
    component of every particle (defaults to what ``set_state`` was given).
    Extra keywords set the header fields of :class:`StateFile`."""
    p = system.params
    if p.n_components == 0:
        raise ValueError("per-particle radius mode has no component table to save")
    st = system.get_state()
    comp = np.asarray(system.comp if comp is None else comp, dtype=np.int32)
    counts = np.bincount(comp, minlength=len(components))
    comps = [ComponentRecord(int(counts[i]), k.radius, k.density, k.stiffness,
                             k.shear_stiffness, k.mass, k.inertia)
             for i, k in enumerate(components)]
    wl = system.walls() if p.n_walls else {"position": [], "velocity": []}
    walls = []
    for j in range(p.n_walls):
        cw = p.walls[j]
        walls.append(WallRecord(int(cw.shape), cw.l1, cw.l2, cw.l3, np.array(cw.u),
                                np.array(cw.w), np.array(cw.n), np.array(wl["position"][j]),
                                np.array(wl["velocity"][j]), np.array(cw.omega),
                                float(wall_stiffness[j][0]), float(wall_stiffness[j][1])))
    L, T, M = scales
    cfg = Configuration(L, T, M, float(step) * p.time_step, np.array(list(p.lbox)), comps,
                        walls, comp, st["pos"], st["vel"], st["omega"])
    _, trav, cs = system.get_cells()
    prev, ipc = system.get_integration()
    if "rng" not in header:  # the pouring generator (aam, Dummy, iix, iiy, iik)
        r = system.rng()
        header["rng"] = (r["aam"], r["dummy"], r["iix"], r["iiy"], r["iik"])
    return StateFile(cfg, trav, cs, ipc, prev, system.get_contacts(), step + 1, system.ncol(),
                     **header)


def params_with_walls(params, state: StateFile):
    """A copy of ``params`` whose walls are those of the state file (moving
    walls are saved where they were)."""
    import copy
    q = copy.deepcopy(params)
    if len(state.config.walls) != q.n_walls:
        raise ValueError("the state file has another number of walls")
    for j, x in enumerate(state.config.walls):
        cw = q.walls[j]
        if int(cw.shape) != x.shape:
            raise ValueError(f"wall {j + 1} has another shape in the state file")
        cw.l1, cw.l2, cw.l3 = x.l1, x.l2, x.l3
        for k in range(3):
            cw.u[k], cw.w[k], cw.n[k] = x.u[k], x.w[k], x.n[k]
            cw.position[k], cw.velocity[k], cw.omega[k] = x.position[k], x.velocity[k], x.omega[k]
    return q


def restore(system, state: StateFile) -> int:
    """ReadState into ``system`` (created from :func:`params_with_walls`):
    particles, cell lists, ring, contacts and Ncol.  Returns InitialStep."""
    c = state.config
    if len(c.components) != system.params.n_components:
        raise ValueError("the state file has another number of components")
    system.set_state(c.pos, c.vel, c.omega, comp=c.index)
    system.set_cells(state.traversal, state.cell_start)
    if system.nprev > 0:
        system.set_integration(state.previous, state.ipc)
    ct = state.contacts
    system.set_contacts(ct["imin"], ct["imax"], ct["ft"], ct["vt"], ct["ip"], ct["iw"],
                        ct["ftw"], ct["vtw"])
    system.set_ncol(state.ncol)
    aam, dummy, iix, iiy, iik = state.rng
    system.set_rng(aam, dummy, iix, iiy, iik)
    return int(state.initial_step)
