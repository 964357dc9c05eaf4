"""Host-side parameter derivation (not a kernel).

Restates, for the C-ABI's ``dem_params``:
  * ``CalculateProperties`` (src/DEM.f90:245-356): component mass/inertia,
    series springs ``Kn = ki*kj/(ki+kj)`` (``Kn(i,i) = 0.5*ki``), effective
    masses, damping from restitution ``gamma = -2 ln e / sqrt(ln^2 e + pi^2)``,
    ``Yn = gamma*sqrt(Meff*Kn)``, the minimum collision time;
  * ``ScaleVariables`` (src/DEM.f90:807-866): length = smallest diameter,
    mass = smallest mass, time = minimum collision time;
  * ``InitializeForce`` (src/MForces.f90:54-87): ``MinDij``, ``InvMass``,
    ``EffectiveMass``, ``MuSq``;
  * ``GramSchmidt`` + ``N = U x W`` for walls (src/MUtil.f90:163-171,
    src/DEM.f90:504-505).

Two entry points:
  * :func:`component_params` -- the reference's discrete components, taking
    values directly in the units the caller wants to simulate in
    (``scale=False``) or in SI to be scaled exactly as the reference does
    (``scale=True``);
  * :func:`per_particle_params` -- continuous polydispersity (per-particle
    radius, one material), the extension described in the C header.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._abi import (MAX_COMPONENTS, MAX_WALLS, POUR_CIRCLE, POUR_RECTANGLE,  # noqa: F401
                   PREC_FP64, PREC_MIXED, WALL_CONE, WALL_RECTANGLE, DemParams, DemWall)

PI = 3.141592653589793238  # the reference's literal (src/DEM.f90:249)


def gamma_from_restitution(e: float) -> float:
    """Gamma = -2*log(E)/sqrt(log(E)**2 + Pi**2) (src/DEM.f90:289-290)."""
    le = math.log(e)
    return -2.0 * le / math.sqrt(le * le + PI * PI)


def gram_schmidt(u, w):
    """GramSchmidt (src/MUtil.f90:163-171) and N = U x W."""
    u = np.asarray(u, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    u = u / math.sqrt(float(((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2])))
    d = (u[0] * w[0] + u[1] * w[1]) + u[2] * w[2]
    w = w - d * u
    w = w / math.sqrt(float(((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2])))
    n = np.array([u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2],
                  u[0] * w[1] - u[1] * w[0]])
    return u, w, n


@dataclass
class Wall:
    """A wall as read by ReadSpecifications (src/DEM.f90:474-505).

    ``l1``/``l2``/``l3`` are the full lengths as written in the input file;
    they are halved on conversion, as the reference does.
    """

    shape: int
    l1: float
    l2: float
    l3: float
    stiffness: float
    shear_stiffness: float
    position: tuple
    u: tuple
    w: tuple
    velocity: tuple = (0.0, 0.0, 0.0)
    omega: tuple = (0.0, 0.0, 0.0)

    def to_c(self, length_scale: float = 1.0, time_scale: float = 1.0) -> DemWall:
        u, w, n = gram_schmidt(self.u, self.w)
        c = DemWall()
        c.shape = self.shape
        c.l1 = 0.5 * self.l1 / length_scale
        c.l2 = 0.5 * self.l2 / length_scale
        c.l3 = 0.5 * self.l3 / length_scale
        for k in range(3):
            c.u[k] = u[k]
            c.w[k] = w[k]
            c.n[k] = n[k]
            c.position[k] = self.position[k] / length_scale
            c.velocity[k] = self.velocity[k] * time_scale / length_scale
            c.omega[k] = self.omega[k]
        return c


def rectangle(center, half_u: float, half_w: float, u=(1.0, 0.0, 0.0), w=(0.0, 1.0, 0.0),
              stiffness: float = 1.0, shear_stiffness: float = 1.0) -> Wall:
    """A flat rectangular wall centred at ``center`` spanning +-half_u, +-half_w."""
    return Wall(WALL_RECTANGLE, 2.0 * half_u, 2.0 * half_w, 0.0, stiffness, shear_stiffness,
                tuple(center), tuple(u), tuple(w))


def cone(center, length: float, diameter_a: float, diameter_p: float, u=(0.0, 0.0, 1.0),
         w=(1.0, 0.0, 0.0), stiffness: float = 1.0, shear_stiffness: float = 1.0) -> Wall:
    """A conic frustum wall (Overlap's Cone branch, src/MConfig.f90:751-793):
    axis ``u`` through ``center``, ``length`` along it, end diameters
    ``diameter_a`` (at the -u end) and ``diameter_p`` (at the +u end), as an
    input file gives them (halved on conversion)."""
    return Wall(WALL_CONE, length, diameter_a, diameter_p, stiffness, shear_stiffness,
                tuple(center), tuple(u), tuple(w))


def wall_motion(position, amplitude, frequency, phase, scales: "Scales | None" = None) -> dict:
    """WM(j) of a wall at ``position`` that oscillates with ``amplitude``,
    ``frequency`` (>= 0) and phase fraction ``phase`` per axis, derived as the
    input reader does (src/DEM.f90:719-733) and, with ``scales``, scaled like
    ScaleVariables (src/DEM.f90:841-847).  The record for
    :meth:`DEMSystem.set_wall_motion`."""
    two_pi = 2.0 * PI
    tpf = [two_pi * float(f) for f in frequency]
    if any(f < 0.0 for f in frequency):
        raise ValueError("wall frequencies cannot be negative")
    ph = [two_pi * float(x) for x in phase]
    amp = [float(a) for a in amplitude]
    m = {"two_pi_frequency": tpf, "phase_angle": ph, "amplitude": amp,
         "velocity_amplitude": [-f * a for f, a in zip(tpf, amp)],
         "constant_factor": [float(x) - a * math.cos(q) for x, a, q in zip(position, amp, ph)]}
    if scales is not None:
        L, T = scales.length, scales.time
        m["constant_factor"] = [x / L for x in m["constant_factor"]]
        m["amplitude"] = [x / L for x in m["amplitude"]]
        m["velocity_amplitude"] = [x * T / L for x in m["velocity_amplitude"]]
        m["two_pi_frequency"] = [x * T for x in m["two_pi_frequency"]]
    return m


def fluid(viscosity: float, flow_rate: float, levels: int, density: float, comp_density,
          scales: "Scales | None" = None):
    """FluidFlow settings (ReadFluidSpecifications, src/mFluid.f90:27-52):
    viscosity, volumetric flow rate, NL levels, the fluid's and the
    components' densities; with ``scales`` converted like
    ScaleFluidProperties/ScaleVariables (src/mFluid.f90:56-68,
    src/DEM.f90:826-858)."""
    from ._abi import DemFluid
    f = DemFluid()
    L = scales.length if scales is not None else 1.0
    M = scales.mass if scales is not None else 1.0
    T = scales.time if scales is not None else 1.0
    f.viscosity = viscosity * L * T / M
    f.flow_rate = flow_rate * T / L ** 3
    f.density = density * L ** 3 / M
    for k, d in enumerate(comp_density):
        f.comp_density[k] = d * L ** 3 / M
    f.levels = int(levels)
    return f


def pouring(target_number, shape: int, size, max_attempts: int, interval: float,
            time_step: float, scales: "Scales | None" = None):
    """Pouring settings as ReadPouringFile and CalculateProperties derive them
    (src/DEM.f90:745-800, 346, 861): ``interval`` is PouringInterval (time),
    IPouring = max(1, nint(interval/time_step)); ``size`` the rectangle sides
    or the circle diameter; with ``scales`` the size is scaled like
    ScaleVariables, and the new spheres get the reference's initial velocity
    -1e-4*LengthScale/TimeScale (src/MDEM.f90:522)."""
    from ._abi import DemPouring
    p = DemPouring()
    p.interval = max(1, int(math.floor(interval / time_step + 0.5)))  # nint, positive
    p.shape = int(shape)
    p.max_attempts = int(max_attempts)
    for k, t in enumerate(target_number):
        if t < 0:
            raise ValueError("target numbers cannot be negative")
        p.target_number[k] = int(t)
    L = scales.length if scales is not None else 1.0
    for k, s in enumerate(size):
        p.size[k] = float(s) / L
    p.velocity_z = -1e-4 * (scales.length / scales.time if scales is not None else 1.0)
    return p


@dataclass
class Component:
    number: int
    diameter: float
    density: float
    stiffness: float
    shear_stiffness: float


@dataclass
class Scales:
    length: float = 1.0
    mass: float = 1.0
    time: float = 1.0
    min_collision_time: float = float("nan")


def _fill_common(p: DemParams, lbox, pbc, gravity, time_step, method_order, euler_intervals,
                 max_ncell, precision, hist_capacity):
    for k in range(3):
        p.lbox[k] = float(lbox[k])
        p.pbc[k] = 1 if pbc[k] else 0
        p.gravity[k] = float(gravity[k])
    p.time_step = float(time_step)
    p.method_order = int(method_order)
    p.euler_intervals = int(euler_intervals)
    p.max_ncell = int(max_ncell)
    p.precision = int(precision)
    p.hist_capacity = int(hist_capacity)


def component_params(components, walls, en, et, mu, enw, etw, muw, *, lbox, pbc, gravity,
                     time_step=None, method_order=4, euler_intervals=100, max_ncell=30000,
                     min_steps_per_collision=None, total_time=None, fluid_density=0.0,
                     scale=False, precision=PREC_FP64, hist_capacity=16):
    """Component-table parameters (src/DEM.f90:245-356, 807-866).

    ``en/et/mu`` are NC x NC, ``enw/etw/muw`` NC x NW.  With ``scale=False``
    the inputs are taken as already expressed in simulation units and
    ``time_step`` must be given.  With ``scale=True`` the SI inputs are scaled
    like ScaleVariables and the time step is derived from
    ``min_steps_per_collision`` and ``total_time`` like CalculateProperties.
    Returns ``(DemParams, Scales)``.
    """
    nc = len(components)
    nw = len(walls)
    if not 1 <= nc <= MAX_COMPONENTS or nw > MAX_WALLS:
        raise ValueError("too many components or walls")
    en = np.asarray(en, float).reshape(nc, nc)
    et = np.asarray(et, float).reshape(nc, nc)
    mu = np.asarray(mu, float).reshape(nc, nc)
    enw = np.asarray(enw, float).reshape(nc, nw) if nw else np.zeros((nc, 0))
    etw = np.asarray(etw, float).reshape(nc, nw) if nw else np.zeros((nc, 0))
    muw = np.asarray(muw, float).reshape(nc, nw) if nw else np.zeros((nc, 0))
    radius = [0.5 * c.diameter for c in components]
    density = [c.density for c in components]
    stiff = [c.stiffness for c in components]
    shear = [c.shear_stiffness for c in components]
    # Component%Mass = 4*Pi/3*R**3*Density ; Inertia = 2/5*Mass*R**2
    mass = [4.0 * PI / 3.0 * (r * r * r) * d for r, d in zip(radius, density)]
    inertia = [2.0 / 5.0 * m * (r * r) for m, r in zip(mass, radius)]
    meff = np.zeros((nc, nc))
    kn = np.zeros((nc, nc))
    kt = np.zeros((nc, nc))
    for i in range(nc):
        meff[i, i] = 0.5 * mass[i]
        kn[i, i] = 0.5 * stiff[i]
        kt[i, i] = 0.5 * shear[i]
        for j in range(i + 1, nc):
            meff[i, j] = meff[j, i] = mass[i] * mass[j] / (mass[i] + mass[j])
            kn[i, j] = kn[j, i] = stiff[i] * stiff[j] / (stiff[i] + stiff[j])
            kt[i, j] = kt[j, i] = shear[i] * shear[j] / (shear[i] + shear[j])
    gn = np.vectorize(gamma_from_restitution)(en)
    gt = np.vectorize(gamma_from_restitution)(et)
    yn = gn * np.sqrt(meff * kn)
    yt = gt * np.sqrt(meff * kt)
    meffw = np.zeros((nc, nw))
    knw = np.zeros((nc, nw))
    ktw = np.zeros((nc, nw))
    for i in range(nc):
        for j in range(nw):
            meffw[i, j] = mass[i]
            knw[i, j] = stiff[i] * walls[j].stiffness / (stiff[i] + walls[j].stiffness)
            ktw[i, j] = shear[i] * walls[j].shear_stiffness / (shear[i] + walls[j].shear_stiffness)
    gnw = np.vectorize(gamma_from_restitution)(enw) if nw else np.zeros((nc, 0))
    gtw = np.vectorize(gamma_from_restitution)(etw) if nw else np.zeros((nc, 0))
    ynw = gnw * np.sqrt(meffw * knw) if nw else np.zeros((nc, 0))
    ytw = gtw * np.sqrt(meffw * ktw) if nw else np.zeros((nc, 0))
    tcs = [np.min(meff / np.sqrt(4.0 * meff * kn - yn ** 2))]
    if nw:
        tcs.append(np.min(meffw / np.sqrt(4.0 * meffw * knw - ynw ** 2)))
    min_collision_time = 2.0 * PI * min(tcs)

    sc = Scales(min_collision_time=float(min_collision_time))
    lbox = [float(x) for x in lbox]
    grav = [float(x) for x in gravity]
    if scale:
        if min_steps_per_collision is None or total_time is None:
            raise ValueError("scale=True needs min_steps_per_collision and total_time")
        ts = min_collision_time / min_steps_per_collision
        nsteps = int(round(total_time / ts))
        ts = total_time / nsteps
        L = 2.0 * min(radius)
        M = min(mass)
        T = min_collision_time
        sc = Scales(L, M, T, float(min_collision_time))
        lbox = [x / L for x in lbox]
        radius = [r / L for r in radius]
        mass = [m / M for m in mass]
        density = [d * L ** 3 / M for d in density]
        inertia = [i / (L ** 2 * M) for i in inertia]
        kn = kn * T ** 2 / M
        yn = yn * T / M
        knw = knw * T ** 2 / M
        ynw = ynw * T / M
        kt = kt * T ** 2 / M
        yt = yt * T / M
        ktw = ktw * T ** 2 / M
        ytw = ytw * T / M
        grav = [g * T ** 2 / L for g in grav]
        fluid_density = fluid_density * L ** 3 / M
        time_step = ts / T
    elif time_step is None:
        raise ValueError("time_step is required when scale=False")

    p = DemParams()
    _fill_common(p, lbox, pbc, grav, time_step, method_order, euler_intervals, max_ncell,
                 precision, hist_capacity)
    p.n_components = nc
    p.n_walls = nw
    K = MAX_COMPONENTS
    W = MAX_WALLS
    for i in range(nc):
        p.comp_radius[i] = radius[i]
        p.comp_inv_mass[i] = 1.0 / mass[i]
        p.comp_inv_inertia[i] = 1.0 / inertia[i]
        p.comp_eff_mass[i] = mass[i] * (density[i] - fluid_density) / density[i]
        for j in range(nc):
            md = 2.0 * radius[i] if i == j else radius[i] + radius[j]
            p.min_dij[i * K + j] = md
            p.min_dij_sq[i * K + j] = md * md
            p.kn[i * K + j] = kn[i, j]
            p.yn[i * K + j] = yn[i, j]
            p.kt[i * K + j] = kt[i, j]
            p.yt[i * K + j] = yt[i, j]
            p.mu_sq[i * K + j] = mu[i, j] ** 2
        for j in range(nw):
            p.knw[i * W + j] = knw[i, j]
            p.ynw[i * W + j] = ynw[i, j]
            p.ktw[i * W + j] = ktw[i, j]
            p.ytw[i * W + j] = ytw[i, j]
            p.muw_sq[i * W + j] = muw[i, j] ** 2
    for j, w in enumerate(walls):
        p.walls[j] = w.to_c(sc.length, sc.time) if scale else w.to_c()
    return p, sc


def per_particle_params(*, density, kn, kt, en, et, mu, rmax, lbox, pbc, gravity, time_step,
                        walls=(), knw=(), ktw=(), enw=(), etw=(), muw=(), fluid_density=0.0,
                        method_order=4, euler_intervals=100, max_ncell=30000,
                        precision=PREC_FP64, hist_capacity=16):
    """Per-particle-radius parameters (continuous polydispersity).

    ``kn``/``kt`` are the pair spring constants (the reference's Kn, Kt after
    the series combination); ``knw``/``ktw`` the particle-wall ones.  Damping
    follows the reference rule with the pair's reduced mass.
    """
    nw = len(walls)
    p = DemParams()
    _fill_common(p, lbox, pbc, gravity, time_step, method_order, euler_intervals, max_ncell,
                 precision, hist_capacity)
    p.n_components = 0
    p.n_walls = nw
    p.pp_mass_coef = 4.0 * PI / 3.0 * density
    p.pp_density = density
    p.pp_fluid_density = fluid_density
    p.pp_rmax = rmax
    p.pp_kn = kn
    p.pp_kt = kt
    p.pp_gamma_n = gamma_from_restitution(en)
    p.pp_gamma_t = gamma_from_restitution(et)
    p.pp_mu_sq = mu * mu
    for j in range(nw):
        p.pp_knw[j] = knw[j]
        p.pp_ktw[j] = ktw[j]
        p.pp_gamma_nw[j] = gamma_from_restitution(enw[j])
        p.pp_gamma_tw[j] = gamma_from_restitution(etw[j])
        p.pp_muw_sq[j] = muw[j] * muw[j]
        p.walls[j] = walls[j].to_c()
    return p


def nprev(params: DemParams) -> int:
    return int(params.method_order) - 1
