"""Fluid drag (mFluid: UpdateVelocityField + DragForce, src/mFluid.f90:96-197)
in the oracle, pinned against a Python restatement: spheres that touch
nothing feel gravity, buoyancy and drag only, so their accelerations follow
from the level tables and the drag law alone."""
import math

import numpy as np
import pytest

from dem3d_b200 import configs
from dem3d_b200 import params as P
from tests.oracle_lib import oracle_system

PI = 3.1415926535897932384626433832795


def fluid_case(n=300, levels=40, flow=6.0, seed=21):
    w = configs.settling(n=n, seed=seed, headroom=20.0, sigma_v=0.8, fluid_density=1.0)
    fl = P.fluid(viscosity=0.05, flow_rate=flow, levels=levels, density=1.0,
                 comp_density=[configs.DENSITY])
    return w, fl


def restated_accelerations(w, fl, pos, vel):
    """ComputeAccelerations for spheres with no contacts: (Fg + FD)/m."""
    prm = w.params
    L = list(prm.lbox)
    nl = fl.levels
    area = L[0] * L[1]
    dz = L[2] / nl
    vf0 = fl.flow_rate / area
    h2 = L[2] / 2.0
    R = prm.comp_radius[0]
    vf, ef = [], []
    for k in range(nl + 1):
        zk = -h2 + k * dz
        sa = sb = sc = 0.0
        for i in range(len(pos)):
            d = zk - pos[i][2]
            if d * d < R * R:
                ai = PI * (R * R - d * d)
                sa = sa + ai
                da = ai * fl.comp_density[0]
                sb = sb + da * vel[i][2]
                sc = sc + da
        if sa == 0.0:
            vf.append(vf0)
            ef.append(1.0)
        else:
            es = sa / area
            ef.append(1.0 - es)
            vf.append((vf0 - es * (sb / sc)) / ef[-1])
    acc = []
    for i in range(len(pos)):
        jr = (pos[i][2] + h2) / dz
        j = min(max(int(jr), 0), nl - 1)
        vfz = vf[j] + (jr - j) * (vf[j + 1] - vf[j])
        efz = ef[j] + (jr - j) * (ef[j + 1] - ef[j])
        vr = [-vel[i][0], -vel[i][1], vfz - vel[i][2]]
        vra = math.sqrt((vr[0] * vr[0] + vr[1] * vr[1]) + vr[2] * vr[2])
        fd = [0.0, 0.0, 0.0]
        if vra > 0.0:
            re = 2.0 * efz * R * vra * fl.density / fl.viscosity
            nn, n0, x = 3.6, 4.6, 0.0
            while abs(nn - n0) > 1e-8:
                n0 = nn
                x = re / math.pow(efz, nn)
                x75 = math.pow(x, 0.75)
                nn = (4.8 + 0.42 * x75) / (1.0 + 0.175 * x75)
            a = 0.63 + 4.8 / math.sqrt(x)
            cd1 = a * a
            a = 0.63 + 4.8 / math.sqrt(re)
            cd = a * a
            fi = (cd1 / cd) * math.pow(efz, 2.0 * (1.0 - nn))
            s = cd * (PI / 2.0) * R * R * fl.density * vra
            fd = [s * vr[k] * fi for k in range(3)]
        em = prm.comp_eff_mass[0]
        f = [em * prm.gravity[k] + fd[k] for k in range(3)]
        acc.append([f[k] * prm.comp_inv_mass[0] for k in range(3)])
    return np.array(acc), np.array(vf), np.array(ef)


def test_drag_matches_the_restatement():
    w, fl = fluid_case()
    o = oracle_system(w.params)
    o.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    o.initialize_cell_distribution()
    o.set_fluid(fl)
    o.compute_accelerations(update=False)
    assert o.count_contacts() == (0, 0)  # the lattice spheres touch nothing
    want, vf, ef = restated_accelerations(w, fl, w.pos, w.vel)
    np.testing.assert_array_equal(o.get_state()["acc"], want)
    assert np.any(ef < 1.0) and np.any(vf != vf[0])  # the bed shapes the flow


def test_upward_flow_lifts_the_spheres():
    w, fl = fluid_case(flow=0.0)
    still = oracle_system(w.params)
    lifted = oracle_system(w.params)
    for s, f in ((still, fl), (lifted, fluid_case(flow=400.0)[1])):
        s.set_state(w.pos, np.zeros_like(w.vel), w.omega, comp=w.comp)
        s.initialize_cell_distribution()
        s.set_fluid(f)
        s.run(1, 200)
    assert lifted.get_state()["pos"][:, 2].mean() > still.get_state()["pos"][:, 2].mean() + 0.01
