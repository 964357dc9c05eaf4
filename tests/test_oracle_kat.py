"""Known-answer tests pinning the CPU oracle to the reference's model.

No outputs of the reference exist (no tests, no shipped results, no Fortran
compiler here), so the oracle is pinned by closed forms of the reference's own
model: the damping rule of CalculateProperties (src/DEM.f90:288-298) makes a
linear spring-dashpot collision restore the requested restitution coefficient
after a contact time pi/omega_d (MinCollisionTime, src/DEM.f90:330-331);
the Coulomb cap (src/MForces.f90:372-378); the rectangle closest-point
geometry (src/MConfig.f90:717-749); CurrentCell3D (src/MCells.f90:498-513);
Newton's third law of the pair loop (src/MForces.f90:254-259); free flight,
which the Euler start-up and the Adams-Bashforth-Moulton steps integrate
exactly; and a sphere resting on the floor, a damped linear oscillator that
the fourth-order integrator follows at fourth order."""
import math

import numpy as np
import pytest

from dem3d_b200 import params as P
from dem3d_b200.configs import DENSITY, KN, KT, settling
from tests.oracle_lib import oracle_system


def two_body(e=0.8, mu=0.5, v0=1.0, dt=1e-5, order=4, gap=0.01, walls=(), gravity=0.0,
             pbc=(False, False, False)):
    prm, _ = P.component_params(
        [P.Component(2, 1.0, DENSITY, 2 * KN, 2 * KT)], list(walls), [[e]], [[e]], [[mu]],
        [[e] * len(walls)], [[e] * len(walls)], [[mu] * len(walls)], lbox=(10.0, 10.0, 10.0),
        pbc=pbc, gravity=(0.0, 0.0, -gravity), time_step=dt, method_order=order,
        euler_intervals=10)
    pos = np.array([[-0.5 - gap, 0.0, 0.0], [0.5 + gap, 0.0, 0.0]])
    vel = np.array([[0.5 * v0, 0.0, 0.0], [-0.5 * v0, 0.0, 0.0]])
    return prm, pos, vel


def run_collision(e, order=4, dt=1e-5, v0=1.0):
    prm, pos, vel = two_body(e=e, dt=dt, order=order, v0=v0)
    s = oracle_system(prm)
    s.set_state(pos, vel, np.zeros((2, 3)), comp=np.zeros(2, np.int32))
    s.initialize_cell_distribution()
    steps = int(0.05 / dt)
    t_in = t_out = None
    s.run(1, order)  # start-up
    step = order
    for _ in range(steps):
        step += 1
        s.move_particles(step)
        st = s.get_state()
        d = st["pos"][1, 0] - st["pos"][0, 0]
        if t_in is None and d < 1.0:
            t_in = step * dt
        if t_in is not None and d >= 1.0:
            t_out = step * dt
            break
    st = s.get_state()
    vrel = st["vel"][1, 0] - st["vel"][0, 0]
    return vrel, t_in, t_out, prm


@pytest.mark.parametrize("e", [0.5, 0.8, 0.95])
def test_head_on_restitution_and_duration(e):
    vrel, t_in, t_out, prm = run_collision(e)
    # restitution: outgoing relative velocity = e * incoming (1.0)
    assert abs(vrel - e) < 2e-3 * max(e, 0.1), (vrel, e)
    # contact time = pi / omega_d with m_eff = m/2, k = Kn, eta = Yn
    kn = prm.kn[0]
    yn = prm.yn[0]
    meff = 0.5 / prm.comp_inv_mass[0]
    wd = math.sqrt(kn / meff - (yn / (2 * meff)) ** 2)
    tc = math.pi / wd
    assert abs((t_out - t_in) - tc) < 3e-5 + 2e-3 * tc, (t_out - t_in, tc)


def test_momentum_and_third_law():
    rng = np.random.default_rng(5)
    n = 300
    prm = P.per_particle_params(density=DENSITY, kn=KN, kt=KT, en=0.7, et=0.7, mu=0.4,
                                rmax=0.6, lbox=(8.0, 8.0, 8.0), pbc=(True, True, True),
                                gravity=(0, 0, 0), time_step=1e-4)
    radius = rng.uniform(0.4, 0.6, n)
    from dem3d_b200.configs import lattice_positions
    pos = lattice_positions(n, 8.0, rng)
    vel = rng.normal(0, 0.3, (n, 3))
    om = rng.normal(0, 0.3, (n, 3))
    s = oracle_system(prm)
    s.set_state(pos, vel, om, radius=radius)
    s.initialize_cell_distribution()
    m = 4.0 / 3.0 * math.pi * DENSITY * radius ** 3
    p0 = (m[:, None] * vel).sum(0)
    s.compute_accelerations(update=True)
    a = s.get_state()["acc"]
    F = (m[:, None] * a).sum(0)
    assert np.abs(F).max() < 1e-9 * np.abs(m[:, None] * a).max()
    s.run(1, 40)
    p1 = (m[:, None] * s.get_state()["vel"]).sum(0)
    assert np.allclose(p0, p1, atol=1e-9, rtol=0)
    assert s.count_contacts()[0] > 0


def test_force_arrays():
    """orc_compute_forces: the pass's Force and Torque sums obey the third
    law (no walls, no gravity) and give the stored accelerations as F/m and
    T/I."""
    rng = np.random.default_rng(6)
    n = 300
    prm = P.per_particle_params(density=DENSITY, kn=KN, kt=KT, en=0.7, et=0.7, mu=0.4,
                                rmax=0.6, lbox=(8.0, 8.0, 8.0), pbc=(True, True, True),
                                gravity=(0, 0, 0), time_step=1e-4)
    radius = rng.uniform(0.4, 0.6, n)
    from dem3d_b200.configs import lattice_positions
    s = oracle_system(prm)
    s.set_state(lattice_positions(n, 8.0, rng), rng.normal(0, 0.3, (n, 3)),
                rng.normal(0, 0.3, (n, 3)), radius=radius)
    s.initialize_cell_distribution()
    s.run(1, 20)
    f, t = s.compute_forces(update=False)
    assert f.shape == t.shape == (n, 3) and np.abs(f).max() > 0
    assert np.abs(f.sum(0)).max() < 1e-9 * np.abs(f).max()
    m = 4.0 / 3.0 * math.pi * DENSITY * radius ** 3
    inertia = 0.4 * m * radius ** 2
    st = s.get_state()
    np.testing.assert_allclose(st["acc"], f / m[:, None], rtol=1e-13, atol=0)
    np.testing.assert_allclose(st["alpha"], t / inertia[:, None], rtol=1e-13, atol=0)


@pytest.mark.parametrize("en,mu", [(1.0, 0.0), (0.7, 0.4)])
def test_energy_between_collisions(en, mu):
    """A periodic gas without gravity, sampled when no contact is open (no
    elastic energy stored): with e = 1 and no friction the kinetic energy
    (translation + rotation) is conserved to the integrator's accuracy over
    hundreds of collisions; with e < 1 and friction it never rises and has
    fallen by the end."""
    rng = np.random.default_rng(11)
    n, L = 216, 11.0
    prm = P.per_particle_params(density=DENSITY, kn=KN, kt=KT, en=en, et=en, mu=mu, rmax=0.55,
                                lbox=(L, L, L), pbc=(True, True, True), gravity=(0, 0, 0),
                                time_step=1e-4)
    from dem3d_b200.configs import lattice_positions
    s = oracle_system(prm)
    s.set_state(lattice_positions(n, L, rng), rng.normal(0, 1.0, (n, 3)),
                rng.normal(0, 1.0, (n, 3)), radius=rng.uniform(0.45, 0.55, n))
    s.initialize_cell_distribution()
    e0 = s.observables()["kinetic_energy"]
    free = []
    for first in range(1, 16001, 20):
        s.run(first, first + 19)
        if s.count_contacts() == (0, 0):
            free.append(s.observables()["kinetic_energy"] / e0)
    assert s.ncol() > 300 and len(free) > 100
    free = np.array(free)
    if en == 1.0:
        assert np.abs(free - 1.0).max() < 5e-5
    else:
        assert np.diff(free).max() <= 1e-12
        assert free[-1] < 0.8


def test_sliding_sphere_rolls_at_five_sevenths():
    """A sphere launched without spin along a frictional floor (linear
    model, Coulomb sliding): while it slides, friction mu*m*g slows it at
    mu*g and spins it up at 5*mu*g/(2R); it rolls from t* = 2*v0/(7*mu*g) on,
    at v = 5/7 v0 with omega*R = v."""
    mu, g, v0, R, dt = 0.5, 1.0, 1.0, 0.5, 1e-4
    L, lz = 10.0, 4.0
    floor = P.rectangle((0.0, 0.0, -0.5 * lz), L, L, stiffness=2.0 * KN,
                        shear_stiffness=2.0 * KT)
    prm, _ = P.component_params([P.Component(1, 1.0, DENSITY, 2.0 * KN, 2.0 * KT)], [floor],
                                [[0.8]], [[0.8]], [[mu]], [[0.8]], [[0.8]], [[mu]],
                                lbox=(L, L, lz), pbc=(True, True, False),
                                gravity=(0.0, 0.0, -g), time_step=dt)
    s = oracle_system(prm)
    m = 1.0  # d = 1 at DENSITY
    s.set_state(np.array([[0.0, 0.0, -0.5 * lz + R - m * g / KN]]), np.array([[v0, 0.0, 0.0]]),
                np.zeros((1, 3)), comp=np.zeros(1, np.int32))
    s.initialize_cell_distribution()
    t_roll = 2.0 * v0 / (7.0 * mu * g)
    half = int(round(0.5 * t_roll / dt))
    s.run(1, half)
    st = s.get_state()
    assert abs(st["vel"][0, 0] - (v0 - mu * g * half * dt)) < 1e-4
    assert abs(st["omega"][0, 1] - 2.5 * mu * g / R * half * dt) < 1e-4
    s.run(half + 1, int(2.1 * t_roll / dt))
    st = s.get_state()
    assert abs(st["vel"][0, 0] - 5.0 / 7.0 * v0) < 1e-6
    assert abs(st["omega"][0, 1] * R - st["vel"][0, 0]) < 1e-6
    assert abs(st["vel"][0, 1]) < 1e-12 and abs(st["omega"][0, 0]) < 1e-12


def test_coulomb_cap_on_records():
    """Every stored tangential force obeys |FT| <= mu |FN| at storage time:
    check a sliding block of spheres on a frictional floor."""
    w = settling(n=200, seed=3, sigma_v=2.0)
    s = oracle_system(w.params)
    s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    s.initialize_cell_distribution()
    s.run(1, 300)
    c = s.get_contacts()
    assert c["imin"].size + c["ip"].size > 0
    assert np.all(c["imin"] < c["imax"])
    # lists sorted like the reference (by imin, then partner)
    key = c["imin"].astype(np.int64) * 10**6 + c["imax"]
    assert np.all(np.diff(key) > 0)


def test_current_cell_matches_formula():
    w = settling(n=500, seed=11)
    s = oracle_system(w.params)
    s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    s.initialize_cell_distribution()
    ci, tr, cs = s.get_cells()
    nx, ny, nz = s.grid()
    L = np.array(w.info["lbox"])
    N = np.array([nx, ny, nz])
    nbyl = N / L
    i3 = np.clip((nbyl * w.pos + N * 0.5).astype(np.int64), 0, N - 1)
    expect = i3[:, 0] + (i3[:, 1] + i3[:, 2] * ny) * nx
    assert np.array_equal(ci, expect)
    # list order after DistributeParticles3D: decreasing index inside a cell
    for c in range(nx * ny * nz):
        members = tr[cs[c]:cs[c + 1]]
        assert np.all(np.diff(members) < 0)
        assert np.all(ci[members] == c)


@pytest.mark.parametrize("where,expect_overlap", [
    ((0.0, 0.0, 0.3), True),     # face
    ((4.9, 0.0, 0.1), True),     # inside face near edge
    ((5.3, 0.0, 0.1), True),     # past the edge, within radius of it
    ((5.5, 0.0, 0.1), False),    # too far from the edge
    ((5.3, 5.3, 0.05), True),    # corner
])
def test_rectangle_wall_geometry(where, expect_overlap):
    wall = P.rectangle((0.0, 0.0, 0.0), 5.0, 5.0, stiffness=2 * KN, shear_stiffness=2 * KT)
    prm, _ = P.component_params([P.Component(1, 1.0, DENSITY, 2 * KN, 2 * KT)], [wall], [[0.8]],
                                [[0.8]], [[0.5]], [[0.8]], [[0.8]], [[0.5]],
                                lbox=(30.0, 30.0, 30.0), pbc=(False, False, False),
                                gravity=(0, 0, 0), time_step=1e-4)
    s = oracle_system(prm)
    pos = np.array([where], dtype=float)
    s.set_state(pos, np.zeros((1, 3)), np.zeros((1, 3)), comp=np.zeros(1, np.int32))
    s.initialize_cell_distribution()
    s.compute_accelerations(update=True)
    a = s.get_state()["acc"][0]
    # closest point of the rectangle [-5,5]^2 x {0}
    q = np.array([np.clip(where[0], -5, 5), np.clip(where[1], -5, 5), 0.0])
    d = np.array(where) - q
    dist = np.linalg.norm(d)
    if expect_overlap:
        assert dist < 0.5
        kn = prm.knw[0]
        f = kn * (0.5 - dist) * d / dist  # static: pure elastic normal force
        assert np.allclose(a / prm.comp_inv_mass[0], f, rtol=1e-12, atol=1e-9)
    else:
        assert np.all(a == 0.0)


@pytest.mark.parametrize("s_ax, r, expect_overlap", [
    (0.0, 3.2, True),     # inside, against the slanted face
    (-5.2, 2.1, True),    # beyond the narrow end, against its rim
    (5.3, 5.2, True),     # beyond the wide end, against its rim
    (0.0, 1.0, False),    # near the axis
    (6.0, 1.0, False),    # past the end, far from the rim
])
def test_cone_wall_geometry(s_ax, r, expect_overlap):
    """Overlap's Cone branch (src/MConfig.f90:751-793): a resting sphere feels
    the elastic force kn*(R - d) along the line from the closest point of the
    frustum's generatrix segment (axial -5 -> radius 2, +5 -> radius 5)."""
    cone = P.cone((0.0, 0.0, 0.0), 10.0, 4.0, 10.0, stiffness=2 * KN, shear_stiffness=2 * KT)
    prm, _ = P.component_params([P.Component(1, 1.0, DENSITY, 2 * KN, 2 * KT)], [cone], [[0.8]],
                                [[0.8]], [[0.5]], [[0.8]], [[0.8]], [[0.5]],
                                lbox=(30.0, 30.0, 30.0), pbc=(False, False, False),
                                gravity=(0, 0, 0), time_step=1e-4)
    s = oracle_system(prm)
    where = np.array([r, 0.0, s_ax])  # axis z, radial direction x
    s.set_state(where[None, :], np.zeros((1, 3)), np.zeros((1, 3)), comp=np.zeros(1, np.int32))
    s.initialize_cell_distribution()
    s.compute_accelerations(update=True)
    a = s.get_state()["acc"][0]
    A, B, Pt = np.array([-5.0, 2.0]), np.array([5.0, 5.0]), np.array([s_ax, r])
    t = np.clip(np.dot(Pt - A, B - A) / np.dot(B - A, B - A), 0.0, 1.0)
    C = A + t * (B - A)
    q = np.array([C[1], 0.0, C[0]])
    d = where - q
    dist = np.linalg.norm(d)
    if expect_overlap:
        assert dist < 0.5
        f = prm.knw[0] * (0.5 - dist) * d / dist
        assert np.allclose(a / prm.comp_inv_mass[0], f, rtol=1e-12, atol=1e-9)
    else:
        assert dist > 0.5
        assert np.all(a == 0.0)


@pytest.mark.parametrize("order", [2, 3, 4])
def test_free_flight_is_exact(order):
    """Free flight under gravity: the Euler start-up (x += v dt + a dt^2/2,
    src/MDEM.f90:240-252) and the Adams-Bashforth-Moulton steps of order 2
    to 4 (src/MDEM.f90:285-369) integrate a constant acceleration exactly,
    so x(t) = x0 + v0 t - g t^2/2 and v(t) = v0 - g t to rounding.  (The
    initial acceleration is given: MoveParticlesEuler stores Particle's
    acceleration into Previous before it computes one.)"""
    dt, g, steps = 1e-3, 1.0, 400
    prm = P.per_particle_params(density=DENSITY, kn=KN, kt=KT, en=0.8, et=0.8, mu=0.5, rmax=0.5,
                                lbox=(20.0, 20.0, 20.0), pbc=(True, True, True),
                                gravity=(0.0, 0.0, -g), time_step=dt, method_order=order,
                                euler_intervals=10)
    x0 = np.array([[0.3, -0.2, 5.0]])
    v0 = np.array([[0.5, -0.25, 0.75]])
    w0 = np.array([[0.1, 0.2, -0.3]])
    a = np.array([[0.0, 0.0, -g]])
    s = oracle_system(prm)
    s.set_state(x0, v0, w0, radius=np.array([0.5]), acc=a)
    s.initialize_cell_distribution()
    s.run(1, steps)
    st = s.get_state()
    t = steps * dt
    np.testing.assert_allclose(st["pos"], x0 + v0 * t + 0.5 * a * t * t, rtol=0, atol=1e-13)
    np.testing.assert_allclose(st["vel"], v0 + a * t, rtol=0, atol=1e-13)
    np.testing.assert_array_equal(st["omega"], w0)
    np.testing.assert_array_equal(st["acc"], a)


def _resting_sphere_error(e, dt, periods=2.0):
    """A sphere on the floor, displaced upwards by half its equilibrium
    overlap m g / kn and released: in contact throughout, it is the damped
    linear oscillator m u'' + gamma u' + kn u = 0 of the wall's
    spring-dashpot (kn and gamma from CalculateProperties'
    restitution rule, src/DEM.f90:288-298); returns the oracle's deviation
    from the closed form after about `periods` periods, relative to the
    initial displacement."""
    w = settling(n=1, seed=3, dt=dt, e=e, method_order=4, euler_intervals=100)
    prm = w.params
    m = 1.0 / prm.comp_inv_mass[0]
    k, gam, g = prm.knw[0], prm.ynw[0], -prm.gravity[2]
    zeq = prm.walls[0].position[2] + prm.comp_radius[0] - m * g / k
    amp = 0.5 * m * g / k
    pos = w.pos.copy()
    pos[0, 2] = zeq + amp
    s = oracle_system(prm)
    s.set_state(pos, np.zeros((1, 3)), np.zeros((1, 3)), comp=w.comp,
                acc=np.array([[0.0, 0.0, -(k / m) * amp]]))
    s.initialize_cell_distribution()
    w0 = math.sqrt(k / m)
    steps = int(round(periods * 2.0 * math.pi / w0 / dt))
    s.run(1, steps)
    t = steps * dt
    b = gam / (2.0 * m)
    wd = math.sqrt(w0 * w0 - b * b)
    u = amp * math.exp(-b * t) * (math.cos(wd * t) + b / wd * math.sin(wd * t))
    return abs(s.get_state()["pos"][0, 2] - zeq - u) / amp


@pytest.mark.parametrize("e", [1.0, 0.8])
def test_resting_sphere_is_a_damped_oscillator_at_fourth_order(e):
    """The wall contact's normal force, gravity and the fourth-order
    integrator together: the error against the closed form falls by more
    than 16x when the time step halves (fourth order, here 35-56x from
    4e-4 to 2e-4) and is below 5e-6 of the displacement at dt = 2e-4
    (about 50 steps per period)."""
    e1 = _resting_sphere_error(e, 4e-4)
    e2 = _resting_sphere_error(e, 2e-4)
    assert e2 < 5e-6
    assert e1 / e2 > 16.0
