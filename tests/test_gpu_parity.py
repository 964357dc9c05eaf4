"""GPU parity: the CUDA library against the CPU oracle through the C-ABI.

FP64 mode must be bit-identical with the oracle: cell assignment and
traversal order, contact-pair sets and history records, accelerations,
predicted state, ABM ring and trajectories over many steps."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system

pytestmark = pytest.mark.gpu


def make_pair(w, **kw):
    g = DEMSystem(w.params)
    o = oracle_system(w.params)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
        s.initialize_cell_distribution()
    return g, o


def assert_same_state(g, o, what=""):
    a, b = g.get_state(), o.get_state()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what} state.{k}")


def assert_same_predicted(g, o, what=""):
    a, b = g.get_predicted(), o.get_predicted()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what} predicted.{k}")


def assert_same_contacts(g, o, what=""):
    a, b = g.get_contacts(), o.get_contacts()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what} contacts.{k}")


def assert_same_cells(g, o, what=""):
    for x, y, name in zip(g.get_cells(), o.get_cells(), ("cell_index", "traversal", "start")):
        np.testing.assert_array_equal(x, y, err_msg=f"{what} {name}")


def test_initial_distribution_and_one_pass():
    w = configs.settling(n=600, seed=21)
    g, o = make_pair(w)
    assert g.grid() == o.grid()
    assert_same_cells(g, o, "init")
    for s in (g, o):
        s.compute_accelerations(update=True)
    assert_same_state(g, o, "pass")
    assert_same_contacts(g, o, "pass")
    assert g.ncol() == o.ncol()


def test_force_arrays_bit_exact():
    """dem_compute_forces: the Force and Torque sums of a pass, before the
    division by mass and inertia, equal the oracle's bit for bit, on the
    current and on the predicted positions of a settling bed (walls,
    gravity, stored histories)."""
    w = configs.settling(n=600, seed=21)
    g, o = make_pair(w)
    for s in (g, o):
        s.run(1, 60)
    for pred in (False, True):
        (fg, tg), (fo, to) = (s.compute_forces(use_predicted=pred, update=False) for s in (g, o))
        assert np.abs(fg).max() > 0 and np.abs(tg).max() > 0
        np.testing.assert_array_equal(fg, fo, err_msg=f"force predicted={pred}")
        np.testing.assert_array_equal(tg, to, err_msg=f"torque predicted={pred}")
        assert_same_state(g, o, f"state after forces predicted={pred}")
        assert_same_predicted(g, o, f"predicted after forces predicted={pred}")
    assert_same_contacts(g, o, "after force passes")
    for s in (g, o):
        s.run(61, 80)
    assert_same_state(g, o, "run after force passes")


def test_settling_trajectory_bit_exact():
    w = configs.settling(n=400, seed=7, sigma_v=0.5)
    g, o = make_pair(w)
    for s in (g, o):
        s.run(1, 4)  # Euler start-up (3 x 100 passes) + first ABM step
    assert_same_state(g, o, "after start-up")
    assert_same_contacts(g, o, "after start-up")
    np.testing.assert_array_equal(g.logical_ring(), o.logical_ring())
    for step in range(5, 400):
        for s in (g, o):
            s.move_particles(step)
        if step % 50 == 0:
            assert_same_state(g, o, f"step {step}")
            assert_same_predicted(g, o, f"step {step}")
            assert_same_contacts(g, o, f"step {step}")
            assert_same_cells(g, o, f"step {step}")
            np.testing.assert_array_equal(g.logical_ring(), o.logical_ring())
    assert g.ncol() == o.ncol()
    assert g.count_contacts()[0] > 0


def test_floor_contacts_bit_exact():
    """First layer starts in contact with the floor: wall records, wall
    forces and their history through the Euler start-up and ABM steps."""
    w = configs.settling(n=300, seed=17, sigma_v=0.01, first_height=0.47)
    g, o = make_pair(w)
    for s in (g, o):
        s.run(1, 4)
    assert o.count_contacts()[1] > 0
    assert_same_state(g, o, "floor start-up")
    assert_same_contacts(g, o, "floor start-up")
    for s in (g, o):
        s.run(5, 150)
    assert_same_state(g, o, "floor")
    assert_same_contacts(g, o, "floor")
    assert g.ncol() == o.ncol()


def test_graph_run_equals_stepwise():
    w = configs.settling(n=300, seed=8, sigma_v=0.5)
    g1, o = make_pair(w)
    g2 = DEMSystem(w.params)
    g2.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    g2.initialize_cell_distribution()
    g1.run(1, 203)          # graphs of 4 steps + remainder
    o.run(1, 203)
    g2.run(1, 4)
    for step in range(5, 204):
        g2.move_particles(step)
    assert_same_state(g1, g2, "graph vs stepwise")
    assert_same_state(g1, o, "graph vs oracle")
    assert_same_contacts(g1, o, "graph vs oracle")
    assert g1.ncol() == o.ncol() == g2.ncol()


def test_dense_polydisperse_bit_exact():
    w = configs.dense_packing(n=3000, phi=0.55, seed=31, relax_steps=0)
    g, o = make_pair(w)
    for s in (g, o):
        s.compute_accelerations(update=True)
    assert_same_state(g, o, "pass")
    assert_same_contacts(g, o, "pass")
    for s in (g, o):
        s.run(1, 60)
    assert_same_state(g, o, "60 steps")
    assert_same_contacts(g, o, "60 steps")
    assert_same_cells(g, o, "60 steps")
    assert g.ncol() == o.ncol()


def test_history_capacity_growth_is_transparent():
    """Tables starting at one record per particle must grow and give the
    same result as the oracle (the overflowing pass is re-run)."""
    w = configs.dense_packing(n=2000, phi=0.55, seed=32, relax_steps=0)
    w.params.hist_capacity = 1
    g, o = make_pair(w)
    for s in (g, o):
        s.run(1, 30)
    assert g.pass_stats()["hist_capacity"] > 1
    assert_same_state(g, o, "grown")
    assert_same_contacts(g, o, "grown")
    assert g.ncol() == o.ncol()


def test_contacts_roundtrip_and_import():
    w = configs.dense_packing(n=1500, phi=0.5, seed=33, relax_steps=0)
    g, o = make_pair(w)
    o.run(1, 10)
    c = o.get_contacts()
    st = o.get_state()
    prev, ipc = o.get_integration()
    g.set_state(st["pos"], st["vel"], st["omega"], radius=w.radius, acc=st["acc"],
                alpha=st["alpha"])
    g.set_integration(prev, ipc)
    g.set_contacts(c["imin"], c["imax"], c["ft"], c["vt"], c["ip"], c["iw"], c["ftw"], c["vtw"])
    assert_same_contacts(g, o, "import")
    # the cell lists are rebuilt from scratch on both sides
    o2 = oracle_system(w.params)
    o2.set_state(st["pos"], st["vel"], st["omega"], radius=w.radius, acc=st["acc"],
                 alpha=st["alpha"])
    o2.set_integration(prev, ipc)
    o2.set_contacts(c["imin"], c["imax"], c["ft"], c["vt"], c["ip"], c["iw"], c["ftw"], c["vtw"])
    for s in (g, o2):
        s.initialize_cell_distribution()
        for step in range(11, 31):
            s.move_particles(step)
    assert_same_state(g, o2, "resumed")
    assert_same_contacts(g, o2, "resumed")


def test_escape_detection():
    """Particles outside +-L/2 after the corrector (UpdateParticleList's test,
    src/MDEM.f90:624-625) are counted, not removed, when removal is off."""
    w = configs.settling(n=100, seed=9, headroom=2.0, sigma_v=30.0)
    g, o = make_pair(w)
    for s in (g, o):
        s.set_particle_removal(False)
        s.run(1, 50)
    assert_same_state(g, o, "escape")
    st = o.get_state()
    L = np.array(w.info["lbox"])
    out = np.any((st["pos"] > 0.5 * L) | (st["pos"] < -0.5 * L), axis=1)
    assert g.escaped() == int(out.sum()) == o.escaped()


def test_observables_match_oracle():
    """Energies, bed packing fraction and height, contacts of the last pass,
    wall forces and pressures: the first layer starts on the floor."""
    w = configs.settling(n=500, seed=12, sigma_v=0.01, first_height=0.47)
    g, o = make_pair(w)
    for s in (g, o):
        s.run(1, 30)
    a, b = g.observables(), o.observables()
    for k in ("kinetic_energy", "potential_energy", "packing_fraction", "mean_coordination",
              "bed_height"):
        assert abs(a[k] - b[k]) <= 1e-12 * max(1.0, abs(b[k])), k
    for k in ("wall_normal_force", "wall_pressure"):
        assert b[k][0] > 0.0, k  # the bed rests on the floor
        np.testing.assert_allclose(a[k], b[k], rtol=1e-12, atol=0.0, err_msg=k)
    for k in ("n_pair_contacts", "n_wall_contacts", "n_pair_records"):
        assert a[k] == b[k], k
    assert 0.2 < b["packing_fraction"] < 0.75 and b["bed_height"] > 1.0


@pytest.mark.slow
def test_large_dense_one_step_bit_exact():
    """200k polydisperse spheres: one full MoveParticles step bit-exact."""
    w = configs.dense_packing(n=200_000, phi=0.55, seed=34, relax_steps=0)
    g, o = make_pair(w)
    for s in (g, o):
        s.compute_accelerations(update=True)
    assert_same_state(g, o, "200k pass")
    assert_same_contacts(g, o, "200k pass")


def test_bidisperse_walls_bit_exact():
    """Two components (d = 1 and 3) in a box closed by a floor and four side
    walls: component tables, rectangle faces/edges/corners, no periodic axis."""
    w = configs.bidisperse_settling(n=3000, width=24.0, headroom=6.0, sigma_v=0.5)
    g, o = make_pair(w)
    for s in (g, o):
        s.run(1, 400)
    assert o.count_contacts()[1] > 0
    assert_same_state(g, o, "bidisperse")
    assert_same_contacts(g, o, "bidisperse")
    assert_same_cells(g, o, "bidisperse")
    assert g.ncol() == o.ncol()


def test_cone_hopper_bit_exact():
    """Spheres falling into a conic hopper (Cone wall + floor): wall contacts
    through Overlap's Cone branch (src/MConfig.f90:751-793)."""
    w = configs.hopper(n=600, seed=1005)
    g, o = make_pair(w)
    for s in (g, o):
        s.run(1, 800)
    assert_same_state(g, o, "hopper")
    assert_same_contacts(g, o, "hopper")
    assert g.ncol() == o.ncol()
    cw = g.get_contacts()
    assert np.count_nonzero(cw["iw"] == 0) > 0  # the cone is touched


def _vibration(w):
    # the cone shakes sideways and vertically, the floor vertically; over 800
    # steps of 1e-4 the phases pass 2*pi (the phase reduction of MoveWalls)
    cone, floor = w.params.walls[0], w.params.walls[1]
    return [configs.P.wall_motion(list(cone.position), (0.01, 0.0, 0.03), (5.0, 0.0, 25.0),
                                  (0.25, 0.0, 0.6)),
            configs.P.wall_motion(list(floor.position), (0.0, 0.0, 0.02), (0.0, 0.0, 20.0),
                                  (0.0, 0.0, 0.1))]


def assert_same_walls(g, o, what=""):
    a, b = g.walls(), o.walls()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what} walls.{k}")


def test_vibrating_hopper_bit_exact():
    """WallsInMovement: MoveWalls after every Euler sub-step and before every
    corrector; graph replays read each step's walls from pinned slots."""
    w = configs.hopper(n=600, seed=1005)
    g, o = make_pair(w)
    for s in (g, o):
        s.set_wall_motion(_vibration(w))
        s.run(1, 800)
    assert_same_state(g, o, "vibrating hopper")
    assert_same_contacts(g, o, "vibrating hopper")
    assert_same_walls(g, o, "vibrating hopper")
    assert g.ncol() == o.ncol()
    cw = g.get_contacts()
    assert np.count_nonzero(cw["iw"] == 0) > 0
    # the motion really moved the walls
    assert g.walls()["position"][1][2] != w.params.walls[1].position[2]


def test_moving_walls_with_table_growth_and_stepwise():
    """Aborted replays (history tables growing from one record) restore the
    walls of the failed step; stepwise calls give the same trajectory."""
    w = configs.hopper(n=400, seed=1008, euler_intervals=10)
    w.params.hist_capacity = 1
    g, o = make_pair(w)
    g2 = DEMSystem(w.params)
    g2.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
    g2.initialize_cell_distribution()
    for s in (g, o, g2):
        s.set_wall_motion(_vibration(w))
    g.run(1, 403)
    o.run(1, 403)
    g2.run(1, 4)
    for step in range(5, 404):
        g2.move_particles(step)
    assert g.pass_stats()["hist_capacity"] > 1
    assert_same_state(g, o, "grown, moving")
    assert_same_contacts(g, o, "grown, moving")
    assert_same_walls(g, o, "grown, moving")
    assert_same_state(g2, o, "stepwise, moving")
    assert_same_walls(g2, o, "stepwise, moving")
    assert g.ncol() == o.ncol() == g2.ncol()
    # stopping: the walls stay where the last step left them
    for s in (g, o):
        s.set_wall_motion(None)
        s.run(404, 420)
    assert_same_state(g, o, "stopped")
    assert_same_walls(g, o, "stopped")
