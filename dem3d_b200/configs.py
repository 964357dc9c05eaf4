"""Seeded synthetic workloads (no dataset exists for this path).

``settling``     -- gravity settling of monodisperse spheres on a jittered
                    lattice in a box periodic in x/y with a frictional floor
                    (the 2,000-sphere CPU-runnable case; any N).
``settling_ensemble`` -- many independent gravity-settling systems of uneven
                    size (log-uniform particle counts), radii uniform in
                    [0.45, 0.55], per-system friction and restitution, each
                    in its own 10 x 10 x-y periodic box with a floor.
``dense_packing``-- polydisperse spheres, radii uniform in [0.4, 0.6], fully
                    periodic cube at a given volume fraction (the 1M / 16M
                    cases).  Positions: a jittered cubic lattice filled in a
                    seeded random order (overlaps allowed), then
                    soft-repulsion relaxation (normal spring + strong damping,
                    no friction) run with the library itself, then seeded
                    Gaussian velocities.

Units: the length unit is the (mean) diameter 1, the mass unit the mass of a
diameter-1 sphere (density 6/pi), time such that kn = 1e5 (pair normal
stiffness after the series combination), dt = 1e-4.  The component
stiffness is 2e5 so that Kn(i,i) = 0.5*k = 1e5 (src/DEM.f90:273); kt = 2/7 kn;
wall stiffness 2e5 gives Knw = 1e5; tangential restitution = normal one.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import params as P

DENSITY = 6.0 / math.pi
KN = 1.0e5
KT = 2.0 / 7.0 * KN


@dataclass
class Workload:
    name: str
    params: object
    pos: np.ndarray
    vel: np.ndarray
    omega: np.ndarray
    comp: np.ndarray | None = None
    radius: np.ndarray | None = None
    info: dict | None = None

    @property
    def n(self):
        return self.pos.shape[0]


def settling(n=2000, seed=1000, layer_side=10, dt=1e-4, e=0.8, mu=0.5, gravity=1.0,
             headroom=45.0, method_order=4, euler_intervals=100, max_ncell=30000,
             precision=P.PREC_FP64, sigma_v=0.1, first_height=1.0, fluid_density=0.0):
    """Monodisperse gravity settling (d = 1, m = 1).

    ``layer_side`` x ``layer_side`` spheres per layer at xy spacing 1.0 in a
    ``layer_side``-wide periodic box, layers at heights 1, 3, 5, ... above the
    floor.  Jitter: U(+-0.05) per particle in z and a rigid U(+-0.05) xy shift
    per layer (a per-particle xy jitter at spacing = diameter would start
    with overlaps of up to 0.1, i.e. 1e4-force kicks).
    """
    rng = np.random.default_rng(seed)
    per_layer = layer_side * layer_side
    n_layers = (n + per_layer - 1) // per_layer
    bed = 2.0 * n_layers
    lz = bed + headroom
    L = float(layer_side)
    pos = np.empty((n, 3))
    k = 0
    for layer in range(n_layers):
        sx, sy = rng.uniform(-0.05, 0.05, size=2)
        for iy in range(layer_side):
            for ix in range(layer_side):
                if k >= n:
                    break
                x = -0.5 * L + 0.5 + ix + sx
                y = -0.5 * L + 0.5 + iy + sy
                z = -0.5 * lz + first_height + 2.0 * layer + rng.uniform(-0.05, 0.05)
                pos[k] = (x, y, z)
                k += 1
    vel = rng.normal(0.0, sigma_v, size=(n, 3))
    omega = np.zeros((n, 3))
    comp = np.zeros(n, dtype=np.int32)
    floor = P.rectangle((0.0, 0.0, -0.5 * lz), L, L, stiffness=2.0 * KN,
                        shear_stiffness=2.0 * KT)
    prm, _ = P.component_params(
        [P.Component(n, 1.0, DENSITY, 2.0 * KN, 2.0 * KT)], [floor], [[e]], [[e]], [[mu]],
        [[e]], [[e]], [[mu]], lbox=(L, L, lz), pbc=(True, True, False),
        gravity=(0.0, 0.0, -gravity), time_step=dt, method_order=method_order,
        euler_intervals=euler_intervals, max_ncell=max_ncell, precision=precision,
        fluid_density=fluid_density)
    return Workload("settling", prm, pos, vel, omega, comp=comp,
                    info={"lbox": (L, L, lz), "seed": seed})


def draining_column(n=600, seed=1013, layer_side=8, dt=5e-4, e=0.7, mu=0.5, gravity=10.0,
                    v_down=10.0, sigma_v=0.5, headroom=2.0, method_order=4, euler_intervals=10,
                    max_ncell=30000, precision=P.PREC_FP64):
    """A column of spheres (d = 1) falling out of the bottom of a box with no
    floor: ``layer_side`` x ``layer_side`` per layer at spacing 1, periodic in
    x/y, layers touching (z jitter U(+-0.01)), moving down at ``v_down``.
    Particles leave through z = -lz/2 layer after layer, in contact with the
    layer above, which exercises UpdateParticleList.  Indices grow from the
    top layer to the bottom one and are shuffled within each layer, so the
    last particle often sits next to the one that leaves."""
    rng = np.random.default_rng(seed)
    per_layer = layer_side * layer_side
    n_layers = (n + per_layer - 1) // per_layer
    lz = float(n_layers) + headroom
    L = float(layer_side)
    pos = np.empty((n, 3))
    k = 0
    for layer in range(n_layers):  # top layer first
        sx, sy = rng.uniform(-0.05, 0.05, size=2)
        z0 = 0.5 * lz - 0.5 - 1.0 * layer - 0.5 * headroom
        order = rng.permutation(per_layer)
        for site in order:
            if k >= n:
                break
            ix, iy = site % layer_side, site // layer_side
            pos[k] = (-0.5 * L + 0.5 + ix + sx, -0.5 * L + 0.5 + iy + sy,
                      z0 + rng.uniform(-0.01, 0.01))
            k += 1
    vel = rng.normal(0.0, sigma_v, size=(n, 3))
    vel[:, 2] -= v_down
    comp = np.zeros(n, dtype=np.int32)
    prm, _ = P.component_params(
        [P.Component(n, 1.0, DENSITY, 2.0 * KN, 2.0 * KT)], [], [[e]], [[e]], [[mu]],
        [], [], [], lbox=(L, L, lz), pbc=(True, True, False), gravity=(0.0, 0.0, -gravity),
        time_step=dt, method_order=method_order, euler_intervals=euler_intervals,
        max_ncell=max_ncell, precision=precision)
    return Workload("draining_column", prm, pos, vel, np.zeros((n, 3)), comp=comp,
                    info={"lbox": (L, L, lz), "seed": seed})


def discharge(n=360, seed=1014, e=0.7, mu=0.5, dt=4e-4, gravity=20.0, v_down=6.0,
              sigma_v=0.3, length=10.0, d_out=3.0, d_in=14.0, method_order=4,
              euler_intervals=10, max_ncell=30000, precision=P.PREC_FP64):
    """A conic hopper (Cone wall, axis z, opening ``d_out`` at the bottom)
    emptying out of a box with no floor: the box ends 0.6 below the outlet,
    so the spheres (d = 1) that pass the outlet leave the box while still
    touching the ones above.  The spheres fill the cone from the outlet up on
    a lattice of spacing 1.02, moving down at ``v_down``; indices grow from
    the top layer down and are shuffled within each layer, so the last
    particle usually sits near the outlet too."""
    rng = np.random.default_rng(seed)
    L = d_in + 4.0
    lz = 2.0 * (0.5 * length + 0.6)
    a = 1.02
    layers = []
    z = -0.5 * length + 0.6
    total = 0
    while total < n:
        if z > 0.5 * length - 0.5:
            raise ValueError("the cone holds fewer spheres")
        r_z = 0.5 * d_out + (z + 0.5 * length) / length * 0.5 * (d_in - d_out)
        m = int(r_z / a) + 1
        pts = [(ix * a, iy * a, z) for iy in range(-m, m + 1) for ix in range(-m, m + 1)
               if math.hypot(ix * a, iy * a) < r_z - 0.6]
        layers.append(pts)
        total += len(pts)
        z += a
    pos = []
    for pts in reversed(layers):  # top layer first
        for k in rng.permutation(len(pts)):
            if len(pos) < n:
                pos.append(pts[k])
    pos = np.asarray(pos) + rng.uniform(-0.005, 0.005, size=(n, 3))
    vel = rng.normal(0.0, sigma_v, size=(n, 3))
    vel[:, 2] -= v_down
    cone = P.cone((0.0, 0.0, 0.0), length, d_out, d_in, stiffness=2.0 * KN,
                  shear_stiffness=2.0 * KT)
    prm, _ = P.component_params(
        [P.Component(n, 1.0, DENSITY, 2.0 * KN, 2.0 * KT)], [cone], [[e]], [[e]], [[mu]],
        [[e]], [[e]], [[mu]], lbox=(L, L, lz), pbc=(False, False, False),
        gravity=(0.0, 0.0, -gravity), time_step=dt, method_order=method_order,
        euler_intervals=euler_intervals, max_ncell=max_ncell, precision=precision)
    return Workload("discharge", prm, pos, vel, np.zeros((n, 3)), comp=np.zeros(n, dtype=np.int32),
                    info={"lbox": (L, L, lz), "seed": seed})


def ball_bearings(precision=P.PREC_FP64, pouring_interval=0.5, max_ncell=30000):
    """The reference's shipped example, examples/ball-bearings/ball-bearings.inp
    and ball-bearings.prg, with its values in SI units and scaled as the
    reference scales them (ScaleVariables): an empty 0.11 x 0.11 x 0.05 m box
    with five cone walls (two of them flat discs, one a flat annulus), all
    orbiting on 1 cm circles at 1.5 Hz (WallsInMovement), and 1 cm steel
    spheres poured from a 2 cm circle every ``pouring_interval`` seconds
    (0.5 s in the example) up to 39 spheres, 10 attempts each; e = 0.7,
    mu = 0.3, gravity 9.8 m/s^2, ABM4 with 10 steps per collision and 100
    Euler sub-steps, 30 s simulated.  Returns (Workload with no spheres,
    wall motions, pouring settings, generator seed)."""
    comps = [P.Component(0, 0.01, 7.8e3, 1.e5, 1.e5)]
    # shape 2 = cone: L1 (height), L2, L3 (end diameters), stiffnesses,
    # position, U, W -- the NW rows of the example
    rows = [(0.015, 0.070, 0.070, -0.0165), (0.000, 0.000, 0.070, -0.0240),
            (0.016, 0.072, 0.072, -0.0170), (0.000, 0.000, 0.072, -0.0250),
            (0.000, 0.070, 0.072, -0.0090)]
    walls = [P.cone((0.01, 0.0, z), l1, l2, l3, u=(0.0, 0.0, 1.0), w=(0.0, 1.0, 0.0),
                    stiffness=1.e5, shear_stiffness=1.e5) for l1, l2, l3, z in rows]
    nw = len(walls)
    prm, sc = P.component_params(
        comps, walls, [[0.7]], [[0.7]], [[0.3]], [[0.7] * nw], [[0.7] * nw], [[0.3] * nw],
        lbox=(0.11, 0.11, 0.05), pbc=(False, False, False), gravity=(0.0, 0.0, -9.8),
        method_order=4, euler_intervals=100, max_ncell=max_ncell, min_steps_per_collision=10.0,
        total_time=30.0, fluid_density=0.0, scale=True, precision=precision)
    # V = -2*Pi*A*sin(2*Pi*(f*t + phi)): A = (0.01, 0.01, 0), f = 1.5 Hz, phi = (0, -0.25, 0)
    motion = [P.wall_motion(w.position, (0.01, 0.01, 0.0), (1.5, 1.5, 1.5), (0.0, -0.25, 0.0),
                            scales=sc) for w in walls]
    ts = prm.time_step * sc.time  # the time step in seconds
    pour = P.pouring([39], P.POUR_CIRCLE, (0.02,), 10, pouring_interval, ts, scales=sc)
    empty = np.zeros((0, 3))
    w = Workload("ball_bearings", prm, empty, empty.copy(), empty.copy(),
                 comp=np.zeros(0, dtype=np.int32),
                 info={"scales": sc, "steps": int(round(30.0 / ts))})
    return w, motion, pour, -20


def hopper(n=600, seed=1005, e=0.7, mu=0.5, dt=1e-4, gravity=1.0, length=10.0, d_out=3.0,
           d_in=14.0, method_order=4, euler_intervals=20, precision=P.PREC_FP64,
           sigma_v=1.0, v_radial=3.0, max_ncell=30000):
    """Monodisperse spheres (d = 1) thrown against a conic hopper: a Cone wall
    (axis z, ``length`` long, opening diameters ``d_out`` at the bottom and
    ``d_in`` at the top) above a floor, in a closed (non-periodic) box.  The
    spheres start on a lattice inside the upper part of the cone, moving
    outwards at ``v_radial`` plus N(0, sigma_v^2) noise."""
    rng = np.random.default_rng(seed)
    L = d_in + 4.0
    lz = 3.0 * length
    side = int((0.5 * d_in - 1.0) * 2.0 / 1.1)
    pts = []
    z = 0.5 * length - 1.0
    while len(pts) < n:
        for iy in range(side):
            for ix in range(side):
                x = (ix - 0.5 * (side - 1)) * 1.1
                y = (iy - 0.5 * (side - 1)) * 1.1
                # inside the cone's cross-section at height z, with a margin
                r_z = 0.5 * d_out + (z + 0.5 * length) / length * 0.5 * (d_in - d_out)
                if math.hypot(x, y) < r_z - 0.55 and len(pts) < n:
                    pts.append((x, y, z))
        z += 1.1
    pos = np.asarray(pts) + rng.uniform(-0.03, 0.03, size=(n, 3))
    vel = rng.normal(0.0, sigma_v, size=(n, 3))
    rr = np.hypot(pos[:, 0], pos[:, 1])
    vel[:, 0] += v_radial * pos[:, 0] / np.maximum(rr, 1e-9)
    vel[:, 1] += v_radial * pos[:, 1] / np.maximum(rr, 1e-9)
    cone = P.cone((0.0, 0.0, 0.0), length, d_out, d_in, stiffness=2.0 * KN,
                  shear_stiffness=2.0 * KT)
    floor = P.rectangle((0.0, 0.0, -0.5 * lz + 1.0), 0.5 * L, 0.5 * L, stiffness=2.0 * KN,
                        shear_stiffness=2.0 * KT)
    prm, _ = P.component_params(
        [P.Component(n, 1.0, DENSITY, 2.0 * KN, 2.0 * KT)], [cone, floor], [[e]], [[e]], [[mu]],
        [[e, e]], [[e, e]], [[mu, mu]], lbox=(L, L, lz), pbc=(False, False, False),
        gravity=(0.0, 0.0, -gravity), time_step=dt, method_order=method_order,
        euler_intervals=euler_intervals, max_ncell=max_ncell, precision=precision)
    return Workload("hopper", prm, pos, vel, np.zeros((n, 3)), comp=np.zeros(n, dtype=np.int32),
                    info={"lbox": (L, L, lz), "seed": seed})


def bidisperse_settling(n=4_000_000, seed=1004, width=200.0, ratio=3.0, number_ratio=20,
                        e=0.7, mu=0.5, dt=5e-5, gravity=1.0, headroom=20.0, method_order=4,
                        euler_intervals=100, max_ncell=1 << 30, precision=P.PREC_FP64,
                        sigma_v=0.1):
    """Wide polydispersity: small (d = 1) and large (d = ``ratio``) spheres,
    small:large = ``number_ratio``:1, settling under gravity in a
    ``width`` x ``width`` box closed by a floor and four side walls (five
    rectangles, no periodic axis).  Two components, as the reference models
    discrete sizes.  Initial state: sites of a cubic lattice of spacing
    1.02*``ratio`` filled bottom-up in seeded random order, each site holding
    one large sphere or a 3x3x3 block of small ones (no overlaps)."""
    rng = np.random.default_rng(seed)
    d_l = ratio
    a = 1.02 * d_l
    m_side = int(width / a)                       # sites per row
    n_large = max(1, int(round(n / (number_ratio + 1))))
    n_small = n - n_large
    blocks = (n_small + 26) // 27
    sites = n_large + blocks
    layers = (sites + m_side * m_side - 1) // (m_side * m_side)
    lz = layers * a + headroom
    kind = np.zeros(sites, dtype=np.int8)
    kind[rng.permutation(sites)[:n_large]] = 1    # 1 = large
    pos = []
    comp = []
    left_small = n_small
    for k in range(sites):
        iz, r = divmod(k, m_side * m_side)
        iy, ix = divmod(r, m_side)
        cx = -0.5 * width + (ix + 0.5) * a
        cy = -0.5 * width + (iy + 0.5) * a
        cz = -0.5 * lz + (iz + 0.5) * a
        if kind[k] == 1:
            pos.append((cx, cy, cz))
            comp.append(1)
        else:
            for bz in (-1, 0, 1):
                for by in (-1, 0, 1):
                    for bx in (-1, 0, 1):
                        if left_small == 0:
                            break
                        pos.append((cx + 1.01 * bx, cy + 1.01 * by, cz + 1.01 * bz))
                        comp.append(0)
                        left_small -= 1
    pos = np.asarray(pos, dtype=np.float64)
    comp = np.asarray(comp, dtype=np.int32)
    nn = pos.shape[0]
    order = cell_major_order_box(pos, (width, width, lz), d_l)
    pos, comp = pos[order], comp[order]
    vel = rng.normal(0.0, sigma_v, size=(nn, 3))
    half = 0.5 * width
    zc = 0.0
    hz = 0.5 * lz
    k_w, kt_w = 2.0 * KN, 2.0 * KT
    walls = [
        P.rectangle((0.0, 0.0, -hz), half + 1.0, half + 1.0, (1, 0, 0), (0, 1, 0), k_w, kt_w),
        P.rectangle((-half, 0.0, zc), half + 1.0, hz, (0, 1, 0), (0, 0, 1), k_w, kt_w),
        P.rectangle((half, 0.0, zc), half + 1.0, hz, (0, 1, 0), (0, 0, 1), k_w, kt_w),
        P.rectangle((0.0, -half, zc), half + 1.0, hz, (1, 0, 0), (0, 0, 1), k_w, kt_w),
        P.rectangle((0.0, half, zc), half + 1.0, hz, (1, 0, 0), (0, 0, 1), k_w, kt_w),
    ]
    comps = [P.Component(n_small, 1.0, DENSITY, 2.0 * KN, 2.0 * KT),
             P.Component(n_large, d_l, DENSITY, 2.0 * KN, 2.0 * KT)]
    E = np.full((2, 2), e)
    M = np.full((2, 2), mu)
    prm, _ = P.component_params(
        comps, walls, E, E, M, np.full((2, 5), e), np.full((2, 5), e), np.full((2, 5), mu),
        lbox=(width, width, lz), pbc=(False, False, False), gravity=(0.0, 0.0, -gravity),
        time_step=dt, method_order=method_order, euler_intervals=euler_intervals,
        max_ncell=max_ncell, precision=precision)
    return Workload("bidisperse_settling", prm, pos, vel, np.zeros((nn, 3)), comp=comp,
                    info={"lbox": (width, width, lz), "seed": seed, "n_large": n_large})


@dataclass
class Ensemble:
    """Independent systems for DEMSystem.ensemble: per-system parameters and
    sizes, particle arrays concatenated by system."""
    params: list
    counts: np.ndarray
    pos: np.ndarray
    vel: np.ndarray
    omega: np.ndarray
    radius: np.ndarray
    info: dict

    @property
    def n(self):
        return self.pos.shape[0]

    def system(self, s):
        """(params, pos, vel, omega, radius) of system s alone."""
        o = int(self.counts[:s].sum())
        k = int(self.counts[s])
        return (self.params[s], self.pos[o:o + k], self.vel[o:o + k], self.omega[o:o + k],
                self.radius[o:o + k])

    def shard(self, rank, world):
        """The systems rank `rank` of `world` advances: every world-th system
        from `rank` on (sizes are drawn at random, so interleaving balances
        the particle counts), as an Ensemble of its own."""
        idx = list(range(rank, len(self.counts), world))
        off = np.concatenate([[0], np.cumsum(self.counts)])
        sel = np.concatenate([np.arange(off[k], off[k + 1]) for k in idx]) if idx else \
            np.zeros(0, dtype=np.int64)
        return Ensemble([self.params[k] for k in idx], np.asarray(self.counts)[idx],
                        self.pos[sel], self.vel[sel], self.omega[sel], self.radius[sel],
                        dict(self.info, shard=(rank, world), systems=idx))


def settling_ensemble(n_systems=4096, seed=1003, nmin=200, nmax=20000, width=10.0,
                      rmin=0.45, rmax=0.55, mu_range=(0.2, 0.8), e_range=(0.5, 0.95),
                      dt=1e-4, gravity=1.0, headroom=45.0, method_order=4, euler_intervals=100,
                      max_ncell=30000, precision=P.PREC_FP64, sigma_v=0.1, counts=None):
    """An ensemble of gravity-settling systems (the batched workload).

    Per system s: N_s = round(exp(U[ln nmin, ln nmax])) spheres (or
    ``counts``), radii U[rmin, rmax], mu_s ~ U(mu_range), restitution
    e_s ~ U(e_range) (normal = tangential, particle-particle and
    particle-floor).  Box ``width`` x ``width`` periodic in x/y, floor at the
    bottom; spheres on a lattice of floor(width / 2 rmax) sites per row and
    layers 2 rmax * 1.8 apart, jittered by U(+-0.02) in z and a rigid
    U(+-0.02) xy shift per layer, numbered layer by layer; velocities
    N(0, sigma_v^2)."""
    rng = np.random.default_rng(seed)
    if counts is None:
        counts = np.rint(np.exp(rng.uniform(math.log(nmin), math.log(nmax), n_systems)))
    counts = np.asarray(counts, dtype=np.int64)
    side = int(width / (2.0 * rmax))
    a = width / side
    dz = 1.8 * (2.0 * rmax)
    params, P_, V_, R_ = [], [], [], []
    for s, n in enumerate(counts):
        n = int(n)
        mu = float(rng.uniform(*mu_range))
        e = float(rng.uniform(*e_range))
        per = side * side
        layers = (n + per - 1) // per
        lz = layers * dz + headroom
        k = np.arange(n)
        iz, r = np.divmod(k, per)
        iy, ix = np.divmod(r, side)
        shift = rng.uniform(-0.02, 0.02, size=(layers, 2))
        pos = np.empty((n, 3))
        pos[:, 0] = -0.5 * width + (ix + 0.5) * a + shift[iz, 0]
        pos[:, 1] = -0.5 * width + (iy + 0.5) * a + shift[iz, 1]
        pos[:, 2] = -0.5 * lz + rmax + iz * dz + rng.uniform(-0.02, 0.02, size=n)
        P_.append(pos)
        V_.append(rng.normal(0.0, sigma_v, size=(n, 3)))
        R_.append(rng.uniform(rmin, rmax, size=n))
        floor = P.rectangle((0.0, 0.0, -0.5 * lz), width, width)
        params.append(P.per_particle_params(
            density=DENSITY, kn=KN, kt=KT, en=e, et=e, mu=mu, rmax=rmax,
            lbox=(width, width, lz), pbc=(True, True, False), gravity=(0.0, 0.0, -gravity),
            time_step=dt, walls=[floor], knw=[KN], ktw=[KT], enw=[e], etw=[e], muw=[mu],
            method_order=method_order, euler_intervals=euler_intervals, max_ncell=max_ncell,
            precision=precision))
    pos = np.concatenate(P_)
    return Ensemble(params, counts, pos, np.concatenate(V_), np.zeros_like(pos),
                    np.concatenate(R_), {"seed": seed, "n_systems": len(counts),
                                         "width": width})


def cell_major_order_box(pos, lbox, cutoff):
    """cell_major_order for a rectangular box."""
    L = np.asarray(lbox, dtype=np.float64)
    nc = np.maximum(1, (L / cutoff).astype(np.int64))
    i3 = np.clip(((pos + 0.5 * L) * (nc / L)).astype(np.int64), 0, nc - 1)
    key = i3[:, 0] + nc[0] * (i3[:, 1] + nc[1] * i3[:, 2])
    return np.argsort(key, kind="stable")


def box_for_fraction(radius: np.ndarray, phi: float) -> float:
    vol = float(np.sum(4.0 / 3.0 * math.pi * radius ** 3))
    return (vol / phi) ** (1.0 / 3.0)


def cell_major_order(pos, L, cutoff):
    """Permutation listing particles cell by cell (x fastest) on the cell grid
    the library builds for a cubic box of side L (InitCellStructure3D with
    CutOff = 2*max radius, no cap).  Particle labels are the user's: the
    library keeps them (the reference's sweep order depends on them), so a
    generator that numbers particles cell by cell gives the library's
    label-indexed arrays the same locality as its cell-ordered traversal."""
    nc = max(1, int(L / cutoff))
    i3 = np.clip(((pos + 0.5 * L) * (nc / L)).astype(np.int64), 0, nc - 1)
    key = i3[:, 0] + nc * (i3[:, 1] + nc * i3[:, 2])
    return np.argsort(key, kind="stable")


def lattice_positions(n: int, L: float, rng, jitter=0.05, cutoff=1.2):
    side = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
    a = L / side
    sites = rng.permutation(side ** 3)[:n]
    iz, r = np.divmod(sites, side * side)
    iy, ix = np.divmod(r, side)
    pos = np.stack([ix, iy, iz], axis=1).astype(np.float64) * a + 0.5 * a - 0.5 * L
    pos += rng.uniform(-jitter, jitter, size=pos.shape) * a
    return pos[cell_major_order(pos, L, cutoff)]


def dense_packing_params(radius_max, L, *, e=0.8, mu=0.5, dt=1e-4, method_order=4,
                         euler_intervals=100, max_ncell=1 << 30, precision=P.PREC_FP64,
                         hist_capacity=4):
    return P.per_particle_params(
        density=DENSITY, kn=KN, kt=KT, en=e, et=e, mu=mu, rmax=radius_max, lbox=(L, L, L),
        pbc=(True, True, True), gravity=(0.0, 0.0, 0.0), time_step=dt,
        method_order=method_order, euler_intervals=euler_intervals, max_ncell=max_ncell,
        precision=precision, hist_capacity=hist_capacity)


def relaxed_tile(n_tile, phi, seed, rmin=0.4, rmax=0.6, relax_steps=2000, relax_e=0.1,
                 system_factory=None):
    """A periodic tile of ``n_tile`` spheres relaxed by soft repulsion.

    Radii U[rmin, rmax]; positions on a jittered cubic lattice filled in a
    seeded random order (overlaps allowed); then ``relax_steps`` ABM steps with
    restitution ``relax_e`` and no friction.  The FP64 library and the CPU
    oracle produce the same tile bit for bit, so either may relax it.
    Returns (pos, radius, L_tile)."""
    rng = np.random.default_rng(seed)
    radius = rng.uniform(rmin, rmax, size=n_tile)
    L = box_for_fraction(radius, phi)
    pos = lattice_positions(n_tile, L, rng, cutoff=2.0 * rmax)
    if relax_steps > 0:
        if system_factory is None:
            from .system import DEMSystem
            system_factory = DEMSystem
        rp = dense_packing_params(rmax, L, e=relax_e, mu=0.0)
        s = system_factory(rp)
        try:
            s.set_state(pos, np.zeros((n_tile, 3)), np.zeros((n_tile, 3)), radius=radius)
            s.initialize_cell_distribution()
            s.run(1, relax_steps)
            pos = s.get_state()["pos"]
        finally:
            s.close()
    return pos, radius, L


def tile_count(n, tile):
    k = int(round((n / tile) ** (1.0 / 3.0)))
    return k if k >= 1 and tile * k ** 3 == n else 0


def replicate(pos, radius, L_tile, k, cutoff=1.2):
    """k x k x k periodic copies of a tile, numbered cell by cell."""
    L = k * L_tile
    offs = (np.stack(np.meshgrid(np.arange(k), np.arange(k), np.arange(k), indexing="ij"),
                     axis=-1).reshape(-1, 3) + 0.5) * L_tile - 0.5 * L
    P_ = (pos[None, :, :] + offs[:, None, :]).reshape(-1, 3)
    R_ = np.tile(radius, k ** 3)
    order = cell_major_order(P_, L, cutoff)
    return P_[order], R_[order], L


def dense_packing(n=1_000_000, phi=0.55, seed=1001, rmin=0.4, rmax=0.6, relax_steps=2000,
                  sigma_v=0.1, precision=P.PREC_FP64, max_ncell=1 << 30, system_factory=None,
                  relax_e=0.1, tile=None):
    """Polydisperse periodic packing at volume fraction ``phi``.

    Large systems are built from a relaxed periodic tile of ``tile`` spheres
    (default 8000 when n = 8000*k^3, else the whole system is one tile)
    replicated k^3 times; the velocities are drawn for the whole system.
    Relaxation runs through ``system_factory`` (the CUDA library by default;
    the oracle in the CPU baseline).  ``relax_steps=0`` skips it."""
    if tile is None:
        tile = 8000 if tile_count(n, 8000) else n
    k = tile_count(n, tile)
    if not k:
        raise ValueError(f"n={n} is not tile*k^3 for tile={tile}")
    pos_t, rad_t, L_t = relaxed_tile(tile, phi, seed, rmin, rmax, relax_steps, relax_e,
                                     system_factory)
    pos, radius, L = replicate(pos_t, rad_t, L_t, k, cutoff=2.0 * rmax)
    rng = np.random.default_rng(seed + 7919)
    vel = rng.normal(0.0, sigma_v, size=(n, 3))
    omega = np.zeros((n, 3))
    info = {"L": L, "phi": phi, "seed": seed, "relax_steps": relax_steps, "tile": tile,
            "copies": k ** 3}
    prm = dense_packing_params(rmax, L, precision=precision, max_ncell=max_ncell)
    return Workload("dense_packing", prm, pos, vel, omega, radius=radius, info=info)


# Volume fraction of the jammed workload.  Radii U[0.4, 0.6] jam near 0.64
# without friction; a frictionless relaxation at a volume fraction below that
# ends with almost no contacts (0.55 gives about 0.3 contacts per sphere, 0.62
# about 0.4), so a packing with about six contacts per sphere needs a volume
# fraction above jamming.  Measured on B200 (8000-sphere tiles relaxed 4000
# steps): 0.64 -> 5.6, 0.66 -> 6.7, 0.68 -> 7.4 contacts per sphere.
JAMMED_PHI = 0.65


def jammed_packing(n=1_000_000, phi=JAMMED_PHI, seed=1012, rmin=0.4, rmax=0.6,
                   relax_steps=4000, sigma_v=0.1, precision=P.PREC_FP64, tile=8000,
                   system_factory=None):
    """Polydisperse periodic packing above jamming (about six contacts per
    sphere): a tile compressed to ``phi`` with overlaps and relaxed without
    friction to mechanical equilibrium (restitution 0.1), replicated; the
    measured contact parameters of the dense configurations (kn = 1e5,
    e = 0.8, mu = 0.5) and seeded velocities N(0, sigma_v^2)."""
    w = dense_packing(n=n, phi=phi, seed=seed, rmin=rmin, rmax=rmax, relax_steps=relax_steps,
                      sigma_v=sigma_v, precision=precision, system_factory=system_factory,
                      tile=tile)
    w.name = "jammed_packing"
    return w


def max_overlap(pos, radius, L, sample=200_000):
    """Largest pair overlap (sampled for very large N) via a cell grid."""
    n = pos.shape[0]
    idx = np.arange(n) if n <= sample else np.random.default_rng(0).choice(n, sample, False)
    cs = 1.2
    nc = max(3, int(L / cs))
    cell = np.floor((pos + 0.5 * L) / L * nc).astype(np.int64) % nc
    key = (cell[:, 2] * nc + cell[:, 1]) * nc + cell[:, 0]
    order = np.argsort(key)
    sk = key[order]
    start = np.searchsorted(sk, np.arange(nc ** 3))
    end = np.searchsorted(sk, np.arange(nc ** 3), side="right")
    best = 0.0
    for i in idx[:20000]:
        ci = cell[i]
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    c = (ci + (dx, dy, dz)) % nc
                    k = (c[2] * nc + c[1]) * nc + c[0]
                    js = order[start[k]:end[k]]
                    js = js[js != i]
                    if js.size == 0:
                        continue
                    d = pos[js] - pos[i]
                    d -= L * np.round(d / L)
                    dist = np.sqrt((d * d).sum(1))
                    ov = radius[js] + radius[i] - dist
                    best = max(best, float(ov.max()))
    return best
