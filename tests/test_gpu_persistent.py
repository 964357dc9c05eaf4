"""Persistent chunks and the launch-shape knobs change how kernels are
launched, never a result.

launch_mode 1 runs each 4-step chunk of dem_run as one cooperative launch
whose blocks step through the chunk's 8 force passes (relink, test, pair and
fold phases with grid-wide barriers between them).  The phases are the same
device code as the separate kernels, and the relink and test code is
written with explicitly rounded operations so that the mixed unit's
contraction does not change a contact decision: every trajectory must be
bit-identical to the graph-replayed one (and, in FP64, to the oracle).
Barrier waits are bounded: a barrier that waits for more blocks than were
launched gives up after its timeout and dem_run reports a state error."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200.system import DEMError, DEMSystem
from tests.oracle_lib import oracle_system

pytestmark = pytest.mark.gpu


def _ensemble(precision):
    # uneven sizes, per-system friction and restitution, fast particles
    return configs.settling_ensemble(n_systems=6, nmin=100, nmax=900, seed=11, sigma_v=4.0,
                                     precision=precision, euler_intervals=10)


def _run_ensemble(e, steps, mode):
    s = DEMSystem.ensemble(e.params, e.counts)
    s.set_launch_shape(launch_mode=mode)
    s.set_state(e.pos, e.vel, e.omega, radius=e.radius)
    s.initialize_cell_distribution()
    l0 = s.launch_count()
    s.run(1, steps)
    out = {"state": s.get_state(), "contacts": s.get_contacts(), "ncol": s.ncol(),
           "launches": s.launch_count() - l0, "blocks": s.persistent_blocks()}
    s.close()
    return out


def _same(a, b, what):
    for k in a["state"]:
        np.testing.assert_array_equal(a["state"][k], b["state"][k], err_msg=f"{what} {k}")
    for k in a["contacts"]:
        np.testing.assert_array_equal(a["contacts"][k], b["contacts"][k], err_msg=f"{what} {k}")
    assert a["ncol"] == b["ncol"], what


@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_MIXED])
def test_persistent_ensemble_equals_graph_chunks(precision):
    e = _ensemble(precision)
    steps = 3 + 4 * 20  # Euler start-up, then 20 whole chunks
    g = _run_ensemble(e, steps, 0)
    p = _run_ensemble(e, steps, 1)
    _same(g, p, "persistent vs graph")
    assert len(g["contacts"]["imin"]) > 0
    # one launch per chunk instead of 8 per step (the start-up is the same)
    assert p["blocks"] > 0
    assert g["launches"] - p["launches"] >= 20 * (4 * 8 - 1)


def _hopper_pair(make, mode, precision=P.PREC_FP64):
    w = configs.hopper(n=600, seed=1005)
    w.params.precision = precision
    s = make(w.params)
    if mode is not None:
        s.set_launch_shape(launch_mode=mode)
    s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
    s.initialize_cell_distribution()
    return s


def test_persistent_cone_hopper_equals_oracle():
    """Walls and a cone (the fold's wall branch and per-block wall sums)."""
    g = _hopper_pair(DEMSystem, 1)
    o = _hopper_pair(oracle_system, None)
    for s in (g, o):
        s.run(1, 800)
    a, b = g.get_state(), o.get_state()
    for k in b:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    ca, cb = g.get_contacts(), o.get_contacts()
    for k in cb:
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    assert g.ncol() == o.ncol()
    assert np.count_nonzero(ca["iw"] == 0) > 0  # the cone is touched


def test_persistent_mixed_hopper_equals_graph_chunks():
    out = []
    for mode in (0, 1):
        s = _hopper_pair(DEMSystem, mode, P.PREC_MIXED)
        s.run(1, 800)
        out.append({"state": s.get_state(), "contacts": s.get_contacts(), "ncol": s.ncol()})
        obs = s.observables()
        s.close()
    _same(out[0], out[1], "mixed hopper")
    assert obs["n_wall_contacts"] > 0


def test_persistent_discharge_with_removals_equals_oracle():
    """Spheres leave through the bottom: a chunk stops before the step that
    follows an escape (the relink phase's escape stop), the host removes
    them and the next chunk is recorded for the new count."""
    w = configs.discharge(d_out=5.0, mu=0.2)
    g, o = DEMSystem(w.params), oracle_system(w.params)
    g.set_launch_shape(launch_mode=1)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        s.run(1, 800)
    assert g.n == o.n < w.pos.shape[0]
    a, b = g.get_state(), o.get_state()
    for k in b:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert g.ncol() == o.ncol()
    assert g.removal_stats() == o.removal_stats()


def _dense(precision=P.PREC_FP64):
    pos, rad, L = configs.relaxed_tile(3000, 0.55, 17, relax_steps=100)
    vel = np.random.default_rng(3).normal(0.0, 0.3, (len(rad), 3))
    s = DEMSystem(configs.dense_packing_params(0.6, L, precision=precision))
    s.set_state(pos, vel, np.zeros_like(vel), radius=rad)
    s.initialize_cell_distribution()
    return s


@pytest.mark.parametrize("shape", [(0, 64, 1, 2), (0, 256, 2, 1), (0, 128, 4, 4),
                                   (1, 128, 1, 2), (1, 64, 2, 4)])
@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_MIXED])
def test_launch_shapes_keep_the_trajectory(shape, precision):
    ref = _dense(precision)
    ref.run(1, 43)
    want, cw = ref.get_state(), ref.get_contacts()
    ref.close()
    s = _dense(precision)
    s.set_launch_shape(*shape)
    assert s.launch_shape() == dict(zip(("launch_mode", "test_block", "particles_per_thread",
                                         "pair_waves"), shape))
    s.run(1, 43)
    got, cg = s.get_state(), s.get_contacts()
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=f"{shape} {k}")
    for k in cw:
        np.testing.assert_array_equal(cg[k], cw[k], err_msg=f"{shape} {k}")
    s.close()


def test_launch_shape_rejects_bad_values():
    s = _dense()
    for bad in ((2, 128, 1, 2), (0, 96, 1, 2), (0, 128, 3, 2), (0, 128, 1, 8)):
        with pytest.raises(DEMError):
            s.set_launch_shape(*bad)
    s.close()


def test_barrier_timeout_is_a_state_error():
    """Every barrier waits for one block more than were launched: the first
    wait of every block runs out (200 ms), the launch ends, dem_run reports
    it, and the context takes a new state and runs again."""
    s = _dense()
    s.set_launch_shape(launch_mode=1)
    s.set_persistent_barrier(200.0, 1)
    with pytest.raises(DEMError, match="barrier timed out"):
        s.run(1, 12)
    s.set_persistent_barrier(2000.0, 0)
    ref = _dense()
    ref.run(1, 12)
    want = ref.get_state()
    pos, rad, L = configs.relaxed_tile(3000, 0.55, 17, relax_steps=100)
    vel = np.random.default_rng(3).normal(0.0, 0.3, (len(rad), 3))
    s.set_state(pos, vel, np.zeros_like(vel), radius=rad)
    s.set_contacts(*[np.zeros(0, dtype=t) for t in (np.int32, np.int32)],
                   np.zeros((0, 3)), np.zeros((0, 3)),
                   np.zeros(0, dtype=np.int32), np.zeros(0, dtype=np.int32),
                   np.zeros((0, 3)), np.zeros((0, 3)))
    s.set_ncol(0)
    s.initialize_cell_distribution()
    s.run(1, 12)
    got = s.get_state()
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
