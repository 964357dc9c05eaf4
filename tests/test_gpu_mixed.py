"""Mixed precision (FP32 contact arithmetic) against the FP64 oracle.

Tolerances: per-step force error <= 1e-5 relative, normed by the largest
|acceleration| of the pass (net forces cancel in packings, so a per-particle
relative error is not meaningful); contact-pair sets identical (the overlap
test stays FP64); ensemble observables within 1% after many steps."""
import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from dem3d_b200.system import DEMSystem
from tests.oracle_lib import oracle_system

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def relaxed(n=4000, phi=0.55, seed=41, steps=300):
    """A relaxed polydisperse packing (GPU relaxation, FP64)."""
    pos, rad, L = configs.relaxed_tile(n, phi, seed, relax_steps=steps)
    rng = np.random.default_rng(seed)
    vel = rng.normal(0, 0.1, (n, 3))
    om = rng.normal(0, 0.1, (n, 3))
    return pos, rad, L, vel, om


def params(L, precision):
    return configs.dense_packing_params(0.6, L, precision=precision)


def test_relaxed_tile_gpu_equals_oracle():
    a = configs.relaxed_tile(1000, 0.55, 5, relax_steps=150)
    b = configs.relaxed_tile(1000, 0.55, 5, relax_steps=150, system_factory=oracle_system)
    np.testing.assert_array_equal(a[0], b[0])


def test_mixed_one_pass_error():
    pos, rad, L, vel, om = relaxed()
    n = len(rad)
    o = oracle_system(params(L, P.PREC_FP64))
    o.set_state(pos, vel, om, radius=rad)
    o.initialize_cell_distribution()
    o.run(1, 20)                      # build contact history
    st = o.get_state()
    c = o.get_contacts()
    prev, ipc = o.get_integration()
    m = DEMSystem(params(L, P.PREC_MIXED))
    for s in (m,):
        s.set_state(st["pos"], st["vel"], st["omega"], radius=rad, acc=st["acc"],
                    alpha=st["alpha"])
        s.set_integration(prev, ipc)
        s.set_contacts(c["imin"], c["imax"], c["ft"], c["vt"], c["ip"], c["iw"], c["ftw"],
                       c["vtw"])
        s.initialize_cell_distribution()
    o2 = oracle_system(params(L, P.PREC_FP64))
    o2.set_state(st["pos"], st["vel"], st["omega"], radius=rad, acc=st["acc"], alpha=st["alpha"])
    o2.set_integration(prev, ipc)
    o2.set_contacts(c["imin"], c["imax"], c["ft"], c["vt"], c["ip"], c["iw"], c["ftw"], c["vtw"])
    o2.initialize_cell_distribution()
    (fm, tm), (fo, to) = (s.compute_forces(update=True) for s in (m, o2))
    # the Force and Torque sums themselves (dem_compute_forces)
    for x, y, kk in ((fm, fo, "force"), (tm, to, "torque")):
        err = np.abs(x - y).max() / np.abs(y).max()
        assert err <= FORCE_TOL, (kk, err)
    a, b = m.get_state(), o2.get_state()
    for k, kk in (("acc", "acceleration"), ("alpha", "angular acceleration")):
        scale = np.abs(b[k]).max()
        err = np.abs(a[k] - b[k]).max() / scale
        assert err <= FORCE_TOL, (kk, err)
    ca, cb = m.get_contacts(), o2.get_contacts()
    np.testing.assert_array_equal(ca["imin"], cb["imin"])
    np.testing.assert_array_equal(ca["imax"], cb["imax"])
    scale = np.abs(cb["ft"]).max()
    assert np.abs(ca["ft"] - cb["ft"]).max() <= FORCE_TOL * scale
    assert m.ncol() == o2.ncol()


def test_mixed_long_run_observables():
    pos, rad, L, vel, om = relaxed(n=8000, seed=43)
    res = {}
    for prec in (P.PREC_FP64, P.PREC_MIXED):
        s = DEMSystem(params(L, prec))
        s.set_state(pos, vel, om, radius=rad)
        s.initialize_cell_distribution()
        s.run(1, 1000)
        res[prec] = s.observables()
        s.close()
    a, b = res[P.PREC_MIXED], res[P.PREC_FP64]
    for k in ("kinetic_energy", "mean_coordination", "packing_fraction"):
        assert abs(a[k] - b[k]) <= 0.01 * abs(b[k]), (k, a[k], b[k])


def test_mixed_settling_with_walls():
    w = configs.settling(n=400, seed=19, sigma_v=0.01, first_height=0.47,
                         precision=P.PREC_MIXED)
    m = DEMSystem(w.params)
    wf = configs.settling(n=400, seed=19, sigma_v=0.01, first_height=0.47)
    f = DEMSystem(wf.params)
    for s, ww in ((m, w), (f, wf)):
        s.set_state(ww.pos, ww.vel, ww.omega, comp=ww.comp)
        s.initialize_cell_distribution()
        s.run(1, 4)
    a, b = m.get_state(), f.get_state()
    assert np.abs(a["pos"] - b["pos"]).max() < 1e-6
    assert m.count_contacts()[1] == f.count_contacts()[1] > 0


def test_mixed_history_growth():
    pos, rad, L, vel, om = relaxed(n=2000, seed=44, steps=100)
    p = params(L, P.PREC_MIXED)
    p.hist_capacity = 1
    s = DEMSystem(p)
    s.set_state(pos, vel, om, radius=rad)
    s.initialize_cell_distribution()
    s.run(1, 40)
    q = DEMSystem(params(L, P.PREC_MIXED))
    q.set_state(pos, vel, om, radius=rad)
    q.initialize_cell_distribution()
    q.run(1, 40)
    assert s.pass_stats()["hist_capacity"] > 1
    np.testing.assert_array_equal(s.get_state()["pos"], q.get_state()["pos"])
