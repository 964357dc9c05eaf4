"""Parity at the benchmark configurations' scale and contact density.

The CUDA path against the oracle on the states the benchmark runs on:
  - the 1,000,000-sphere periodic packing built exactly as bench.py builds it
    (relaxed tile x 125, its velocities), one full MoveParticles step in FP64
    from the same mid-run state, bit for bit, and one mixed-precision pass
    within the force tolerance;
  - a jammed polydisperse packing (about six contacts per sphere), FP64 bit
    for bit over several steps and the mixed pass within the tolerance;
  - an ensemble of 64 settling systems with sizes log-uniform in
    [200, 20000], each system compared with the oracle after its bed has
    started to form;
  - a bidisperse box closed by a floor and four side walls, run from rest
    past the impact on the floor.
A mid-run state moves from the GPU to the oracle through the C-ABI's state,
integration ring, contact records and Ncol (the data a checkpoint holds); both
sides then build their cell lists afresh from the positions
(InitializeCellDistribution), so both continue from identical data.

Force tolerance of the mixed path: 1e-5, normed by the largest |value| of the
pass (net forces cancel in packings)."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def transfer(src, dst, radius=None, comp=None, lo=0, hi=None):
    """Particles [lo, hi) of `src` into `dst`, renumbered from 0: state, ring,
    contact records (and Ncol for a whole system); `dst` builds its cell lists
    from the positions."""
    st = src.get_state()
    hi = src.n if hi is None else hi
    sl = slice(lo, hi)
    dst.set_state(st["pos"][sl], st["vel"][sl], st["omega"][sl],
                  comp=None if comp is None else comp[sl],
                  radius=None if radius is None else radius[sl], acc=st["acc"][sl],
                  alpha=st["alpha"][sl])
    prev, ipc = src.get_integration()
    dst.set_integration(prev[:, sl, :], ipc)
    c = src.get_contacts()
    m = (c["imin"] >= lo) & (c["imin"] < hi)
    mw = (c["ip"] >= lo) & (c["ip"] < hi)
    dst.set_contacts(c["imin"][m] - lo, c["imax"][m] - lo, c["ft"][m], c["vt"][m],
                     c["ip"][mw] - lo, c["iw"][mw], c["ftw"][mw], c["vtw"][mw])
    if lo == 0 and hi == src.n:
        dst.set_ncol(src.ncol())
    dst.initialize_cell_distribution()


def compare(g, o, what, lo=0, hi=None):
    hi = g.n if hi is None else hi
    a, b = g.get_state(), o.get_state()
    for k in b:
        np.testing.assert_array_equal(a[k][lo:hi], b[k], err_msg=f"{what} state.{k}")
    ca, cb = g.get_contacts(), o.get_contacts()
    m = (ca["imin"] >= lo) & (ca["imin"] < hi)
    mw = (ca["ip"] >= lo) & (ca["ip"] < hi)
    np.testing.assert_array_equal(ca["imin"][m] - lo, cb["imin"], err_msg=f"{what} imin")
    np.testing.assert_array_equal(ca["imax"][m] - lo, cb["imax"], err_msg=f"{what} imax")
    for k in ("ft", "vt"):
        np.testing.assert_array_equal(ca[k][m], cb[k], err_msg=f"{what} {k}")
    np.testing.assert_array_equal(ca["ip"][mw] - lo, cb["ip"], err_msg=f"{what} ip")
    for k in ("iw", "ftw", "vtw"):
        np.testing.assert_array_equal(ca[k][mw], cb[k], err_msg=f"{what} {k}")


def mixed_force_error(src, params_fp64, params_mixed, radius=None, comp=None):
    """One history-updating force pass from the same state in the oracle
    (FP64) and in the mixed-precision library; returns the relative errors."""
    out = {}
    for name, prm, make in (("fp64", params_fp64, oracle_system),
                            ("mixed", params_mixed, DEMSystem)):
        s = make(prm)
        transfer(src, s, radius=radius, comp=comp)
        f, t = s.compute_forces(update=True)
        out[name] = (f, t, s.get_state())
        s.close()
    err = {}
    for i, k in ((0, "force"), (1, "torque")):
        ref = out["fp64"][i]
        err[k] = float(np.abs(out["mixed"][i] - ref).max() / np.abs(ref).max())
    for k in ("acc", "alpha"):
        ref = out["fp64"][2][k]
        err[k] = float(np.abs(out["mixed"][2][k] - ref).max() / np.abs(ref).max())
    return err


def test_config1_million_spheres_step_bit_exact():
    """The benchmark's 1M-sphere workload: the GPU runs the Euler start-up and
    a few ABM steps, then GPU and oracle each run one MoveParticles step from
    that state; everything must be equal, and the mixed pass's forces within
    the tolerance."""
    w = configs.dense_packing(n=1_000_000, phi=0.55, seed=1001, tile=8000)
    g = DEMSystem(w.params)
    g.set_state(w.pos, w.vel, w.omega, radius=w.radius)
    g.initialize_cell_distribution()
    g.run(1, 8)
    o = oracle_system(w.params)
    transfer(g, o, radius=w.radius)
    g.initialize_cell_distribution()
    compare(g, o, "transfer")
    for s in (g, o):
        s.move_particles(9)
    compare(g, o, "1M step")
    np.testing.assert_array_equal(g.get_cells()[1], o.get_cells()[1])
    assert g.ncol() == o.ncol()
    assert g.count_contacts()[0] > 0.1 * w.n
    o.close()
    pm = configs.dense_packing_params(0.6, w.info["L"], precision=P.PREC_MIXED)
    err = mixed_force_error(g, w.params, pm, radius=w.radius)
    for k, v in err.items():
        assert v <= FORCE_TOL, (k, v)
    g.close()


def test_jammed_packing_bit_exact_and_mixed():
    """A jammed packing (about six contacts per sphere): FP64 bit for bit over
    several steps from the same state, and the mixed pass within tolerance."""
    w = configs.jammed_packing(n=8000 * 27, seed=1012)
    g = DEMSystem(w.params)
    g.set_state(w.pos, w.vel, w.omega, radius=w.radius)
    g.initialize_cell_distribution()
    g.run(1, 6)
    z = g.observables()["mean_coordination"]
    assert z > 5.0, z
    o = oracle_system(w.params)
    transfer(g, o, radius=w.radius)
    g.initialize_cell_distribution()
    for step in range(7, 11):
        for s in (g, o):
            s.move_particles(step)
    compare(g, o, "jammed")
    assert g.ncol() == o.ncol()
    o.close()
    pm = configs.dense_packing_params(0.6, w.info["L"], precision=P.PREC_MIXED)
    err = mixed_force_error(g, w.params, pm, radius=w.radius)
    for k, v in err.items():
        assert v <= FORCE_TOL, (k, v)
    g.close()


def test_ensemble_64_systems_against_oracle():
    """64 settling systems (sizes log-uniform in [200, 20000], per-system
    friction and restitution) in one FP64 context; once the bottom layers
    sit on the floor, every system continues for 4 steps in the ensemble and
    alone in the oracle, and must match bit for bit."""
    e = configs.settling_ensemble(n_systems=64, seed=1003, precision=P.PREC_FP64)
    s = DEMSystem.ensemble(e.params, e.counts)
    s.set_state(e.pos, e.vel, e.omega, radius=e.radius)
    s.initialize_cell_distribution()
    s.run(1, 1500)
    off = np.concatenate([[0], np.cumsum(e.counts)])
    oracles = []
    for k in range(len(e.counts)):
        o = oracle_system(e.system(k)[0])
        o.set_particle_removal(False)  # as in an ensemble
        transfer(s, o, radius=e.radius, lo=off[k], hi=off[k + 1])
        oracles.append(o)
    s.initialize_cell_distribution()
    s.run(1501, 1504)
    walls = 0
    for k, o in enumerate(oracles):
        n0 = o.ncol()
        o.run(1501, 1504)
        compare(s, o, f"system {k}", lo=off[k], hi=off[k + 1])
        assert o.ncol() >= n0
        walls += o.count_contacts()[1]
        o.close()
    assert walls > 0  # the beds are on the floor
    s.close()


def test_bidisperse_walls_past_floor_impact():
    """Bidisperse spheres (d = 1 and 3, 20:1) in a box closed by a floor and
    four side walls, from rest to well past the impact on the floor (gravity
    10: the lowest layer lands after about 1,300 of the 3,000 steps)."""
    w = configs.bidisperse_settling(n=4000, width=24.0, headroom=4.0, sigma_v=0.2,
                                    gravity=10.0)
    g = DEMSystem(w.params)
    o = oracle_system(w.params)
    for s in (g, o):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp, radius=w.radius)
        s.initialize_cell_distribution()
        s.run(1, 3000)
    compare(g, o, "bidisperse")
    assert o.count_contacts()[1] > 100  # resting on the floor and the walls
    assert g.ncol() == o.ncol()
    np.testing.assert_array_equal(g.get_cells()[1], o.get_cells()[1])
