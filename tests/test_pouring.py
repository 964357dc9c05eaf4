"""Pouring (PouringAttempt/PourParticle/InsertParticle, src/DEM.f90:115-123,
src/MDEM.f90:412-561) and its generator ranf (src/MUtil.f90:17-48) in the
oracle, pinned against restatements written here in Python."""
import ctypes as C
import math

import numpy as np
import pytest

from dem3d_b200 import _abi, configs
from dem3d_b200 import params as P
from tests.oracle_lib import load_oracle, oracle_system
from tests.test_particle_removal import neighbourhood


def ranf_py(s):
    """ranf over Python integers: Marsaglia xorshift (logical shifts on 32
    bits) combined with Park-Miller by Schrage's method; aam in float32."""
    IA, IM, IQ, IR = 16807, 2147483647, 127773, 2836
    if s["dummy"] <= 0 or s["iiy"] < 0:
        s["aam"] = float(np.float32(np.nextafter(np.float32(1.0), np.float32(0.0)))
                         / np.float32(IM))
        ad = abs(s["dummy"])
        s["iiy"] = (888889999 ^ ad) | 1
        s["iix"] = 777755555 ^ ad
        s["dummy"] = ad + 1
    x = s["iix"] & 0xFFFFFFFF
    x ^= (x << 13) & 0xFFFFFFFF
    x ^= x >> 17
    x ^= (x << 5) & 0xFFFFFFFF
    s["iix"] = x - (1 << 32) if x >= (1 << 31) else x
    s["iik"] = s["iiy"] // IQ
    s["iiy"] = IA * (s["iiy"] - s["iik"] * IQ) - IR * s["iik"]
    if s["iiy"] < 0:
        s["iiy"] += IM
    return s["aam"] * float((IM & (s["iix"] ^ s["iiy"])) | 1)


@pytest.mark.parametrize("seed", [-1, -12345, -987654321])
def test_ranf_matches_the_restatement(seed):
    lib = load_oracle()
    lib.orc_ranf.argtypes = [C.POINTER(_abi.DemRng), C.c_int32, C.POINTER(C.c_double)]
    r = _abi.DemRng(0.0, seed, -1, -1, 0)
    out = (C.c_double * 2000)()
    lib.orc_ranf(C.byref(r), 2000, out)
    s = {"aam": 0.0, "dummy": seed, "iix": -1, "iiy": -1, "iik": 0}
    want = [ranf_py(s) for _ in range(2000)]
    assert list(out) == want
    assert (r.dummy, r.iix, r.iiy, r.iik) == (s["dummy"], s["iix"], s["iiy"], s["iik"])
    v = np.array(want)
    assert v.min() > 0.0 and v.max() < 1.0 and abs(v.mean() - 0.5) < 0.03


def filling_box(n_start=40, seed=1015, shape=_abi.POUR_RECTANGLE, attempts=30, interval=5):
    """Two components (d = 1 and 1.5) settling in a closed box while spheres
    are poured from the top."""
    rng = np.random.default_rng(seed)
    L, lz = 14.0, 12.0
    walls = [P.rectangle((0.0, 0.0, -0.5 * lz), 0.5 * L, 0.5 * L,
                         stiffness=2.0 * configs.KN, shear_stiffness=2.0 * configs.KT)]
    comps = [P.Component(n_start // 2, 1.0, configs.DENSITY, 2.0 * configs.KN, 2.0 * configs.KT),
             P.Component(n_start - n_start // 2, 1.5, configs.DENSITY, 2.0 * configs.KN,
                         2.0 * configs.KT)]
    prm, _ = P.component_params(comps, walls, [[0.7] * 2] * 2, [[0.7] * 2] * 2, [[0.5] * 2] * 2,
                                [[0.7]] * 2, [[0.7]] * 2, [[0.5]] * 2, lbox=(L, L, lz),
                                pbc=(True, True, False), gravity=(0.0, 0.0, -10.0),
                                time_step=5e-4, method_order=4, euler_intervals=10)
    side = 6
    pos = []
    for k in range(n_start):
        ix, iy, iz = k % side, (k // side) % side, k // (side * side)
        pos.append((-5.0 + 2.0 * ix, -5.0 + 2.0 * iy, -0.5 * lz + 1.0 + 1.6 * iz))
    pos = np.array(pos) + rng.uniform(-0.02, 0.02, (n_start, 3))
    comp = np.array([0] * (n_start // 2) + [1] * (n_start - n_start // 2), np.int32)
    size = (13.0, 13.0) if shape == _abi.POUR_RECTANGLE else (13.0,)
    pour = P.pouring([60, 45], shape, size, attempts, interval * 5e-4, 5e-4)
    return prm, pos, comp, pour


def start(make, prm, pos, comp, pour, seed=-7):
    s = make(prm)
    s.set_state(pos, np.zeros_like(pos), np.zeros_like(pos), comp=comp)
    s.initialize_cell_distribution()
    s.set_pouring(pour)
    s.set_rng(dummy=seed)
    return s


def restated_pour(state, rng, prm, pour, comp_count, grid, pbc):
    """PourParticle over exported state: the point that goes in (or None)."""
    nc = prm.n_components
    nr = [k for k in range(nc) if comp_count[k] < pour.target_number[k]]
    if not nr:
        return None, rng
    j = int(float(len(nr)) * ranf_py(rng))
    radii = [prm.comp_radius[k] for k in range(nc)]
    ibig = int(np.argmax(radii))
    Ri = radii[ibig]
    Di = 2.0 * Ri
    z = 0.5 * prm.lbox[2] - Ri
    nx, ny, nz = grid
    pos, cmp, ci, tr, cs = state
    for _ in range(pour.max_attempts):
        if pour.shape == _abi.POUR_RECTANGLE:
            x = (pour.size[0] - Di) * (ranf_py(rng) - 0.5)
            y = (pour.size[1] - Di) * (ranf_py(rng) - 0.5)
        else:
            rad = 0.5 * ranf_py(rng) * (pour.size[0] - Di)
            ang = 2.0 * 3.1415926535897932384626433832795 * ranf_py(rng)
            x, y = rad * math.sin(ang), rad * math.cos(ang)
        # CurrentCell3D (clamped truncation)
        idx = []
        for v, n, L in ((x, nx, prm.lbox[0]), (y, ny, prm.lbox[1]), (z, nz, prm.lbox[2])):
            k = int(n / L * v + n / 2.0)
            idx.append(min(max(k, 0), n - 1))
        cell = idx[0] + nx * (idx[1] + ny * idx[2])
        ok = True
        for c in neighbourhood(cell, grid, pbc):
            for q in tr[cs[c]:cs[c + 1]]:
                r = [int(pos[q][0] - x), int(pos[q][1] - y), int(pos[q][2] - z)]
                if not float(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) > prm.min_dij_sq[
                        ibig * _abi.MAX_COMPONENTS + cmp[q]]:
                    ok = False
        if ok and z - Ri < -0.5 * prm.lbox[2]:  # the floor is far below the pouring plane
            ok = False
        if ok:
            return (nr[j], x, y, z), rng
    return None, rng


@pytest.mark.parametrize("shape", [_abi.POUR_RECTANGLE, _abi.POUR_CIRCLE])
def test_pour_matches_the_restatement(shape):
    prm, pos, comp, pour = filling_box(shape=shape)
    o = start(oracle_system, prm, pos, comp, pour)
    inserted = 0
    for step in range(1, 121):
        if step < 4 or step % 5:
            o.move_particles(step) if step >= 4 else o.move_particles_euler()
            continue
        ci, tr, cs = o.get_cells()
        st = o.get_state()
        counts = np.bincount(o.comp, minlength=2)
        state = (st["pos"], o.comp, ci, tr, cs)
        want, rng_after = restated_pour(state, dict(o.rng()), prm, pour, counts, o.grid(),
                                        [1, 1, 0])
        n0 = o.n
        got = o.pour_particle()
        assert o.rng() == rng_after
        assert got == (want is not None)
        if got:
            inserted += 1
            assert o.n == n0 + 1
            k, x, y, z = want
            assert o.comp[-1] == k
            np.testing.assert_array_equal(o.get_state()["pos"][-1], [x, y, z])
            np.testing.assert_array_equal(o.get_state()["vel"][-1], [0.0, 0.0, pour.velocity_z])
        o.move_particles(step)
    assert inserted >= 10


def test_run_pours_every_interval():
    prm, pos, comp, pour = filling_box()
    o = start(oracle_system, prm, pos, comp, pour)
    o.run(1, 300)
    # PouringAttempt runs at steps 5, 10, ... of the main loop (not the Euler start-up)
    assert 40 < o.n <= 40 + 300 // 5
    counts = np.bincount(o.comp, minlength=2)
    assert counts[0] <= 60 and counts[1] <= 45
