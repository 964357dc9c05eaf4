"""UpdateParticleList (src/MDEM.f90:612-671) in the oracle, pinned against an
independent restatement written here over the exported state: particles
outside the box are removed highest index first, the last particle takes
each one's place, and the contact lists are cut and renamed as
RemoveParticleFromContactList and ChangeIndexInContactList do
(src/MContacts.f90:173-252, 579-633)."""
import bisect

import numpy as np
import pytest

from dem3d_b200 import configs
from tests.oracle_lib import oracle_system


def neighbourhood(cell, grid, pbc):
    """The cell and its MonteCarlo neighbour cells (NeighbourCells3D,
    src/MCells.f90:353-375, VerifyPBC/ApplyPBC :1030-1052) in list order:
    AddNeighbour prepends (:666-680), so the neighbours come in the reverse
    of the loop order."""
    nx, ny, nz = grid
    iz = cell // (nx * ny)
    iy = cell // nx - iz * ny
    ix = cell - (iy + iz * ny) * nx
    ranges = []
    for c, n, p in ((ix, nx, pbc[0]), (iy, ny, pbc[1]), (iz, nz, pbc[2])):
        lo, hi = -1, 1
        if not p:
            lo = 0 if c == 0 else -1
            hi = 0 if c == n - 1 else 1
        ranges.append((lo, hi))
    out = []
    for kz in range(ranges[2][0], ranges[2][1] + 1):
        for ky in range(ranges[1][0], ranges[1][1] + 1):
            for kx in range(ranges[0][0], ranges[0][1] + 1):
                if kx == ky == kz == 0:
                    continue
                j = [ix + kx, iy + ky, iz + kz]
                for d, (n, p) in enumerate(zip(grid, pbc)):
                    if p:
                        j[d] = 0 if j[d] == n else (n - 1 if j[d] == -1 else j[d])
                out.append(j[0] + nx * (j[1] + ny * j[2]))
    return [cell] + out[::-1]


def restated_removal(state, lbox, grid, pbc, literal=False):
    """UpdateParticleList over plain Python lists (independent of the C code).
    literal: the records particle i inherits keep the reference's append
    order instead of being ordered by partner."""
    pos = [list(p) for p in state["pos"]]
    vel = [list(v) for v in state["vel"]]
    ring = [list(map(list, slot)) for slot in state["prev"]]
    ci = list(state["cell_index"])
    tr, cs = state["traversal"], state["cell_start"]
    cells = [list(tr[cs[k]:cs[k + 1]]) for k in range(len(cs) - 1)]
    ct = state["contacts"]
    n = len(pos)
    pairs = {i: [] for i in range(n)}
    for a, b, f, v in zip(ct["imin"], ct["imax"], ct["ft"], ct["vt"]):
        pairs[int(a)].append([int(b), tuple(f), tuple(v)])
    walls = {i: [] for i in range(n)}
    for a, w, f, v in zip(ct["ip"], ct["iw"], ct["ftw"], ct["vtw"]):
        walls[int(a)].append([int(w), tuple(f), tuple(v)])
    moved = 0
    for i in range(n - 1, -1, -1):
        if not any(pos[i][k] > 0.5 * lbox[k] or pos[i][k] < -0.5 * lbox[k] for k in range(3)):
            continue
        S = [q for c in neighbourhood(ci[i], grid, pbc) for q in cells[c]]
        cells[ci[i]].remove(i)
        for j in S:
            pairs[j] = [r for r in pairs[j] if r[0] != i]
        pairs[i], walls[i] = [], []
        NP = n - 1
        if i != NP:
            pos[i], vel[i] = pos[NP], vel[NP]
            for slot in ring:
                slot[i] = slot[NP]
            c = ci[NP]
            cells[c][cells[c].index(NP)] = i
            ci[i] = c
            first = []
            for j in S:
                lst = pairs[j]
                if not lst or lst[-1][0] != NP:
                    continue
                rec = lst.pop()
                moved += 1
                if j < i:
                    rec[0] = i
                    bisect.insort(lst, rec)
                else:
                    rec[0] = j
                    first.append(rec)
            pairs[i] = first if literal else sorted(first)
            walls[i], walls[NP] = walls[NP], []
            pairs[NP] = []
        n -= 1
        pos, vel, ci = pos[:n], vel[:n], ci[:n]
        ring = [slot[:n] for slot in ring]
    imin = [a for a in range(n) for _ in pairs[a]]
    imax = [r[0] for a in range(n) for r in pairs[a]]
    trav = [q for c in cells for q in c]
    return dict(pos=np.array(pos).reshape(-1, 3), vel=np.array(vel).reshape(-1, 3),
                ring=np.array(ring), cell_index=np.array(ci), traversal=np.array(trav),
                imin=np.array(imin), imax=np.array(imax), moved=moved,
                ft=np.array([r[1] for a in range(n) for r in pairs[a]]).reshape(-1, 3))


def export(s, logical=False):
    """The state, cells, contacts and ABM ring of a system: the ring as stored
    (physical slots) or, to compare two implementations, in ipc order."""
    st = s.get_state()
    ci, tr, cs = s.get_cells()
    prev = s.logical_ring() if logical else s.get_integration()[0]
    return dict(pos=st["pos"], vel=st["vel"], cell_index=ci, traversal=tr, cell_start=cs,
                contacts=s.get_contacts(), prev=prev)


def dense_case(make, seed=51):
    w = configs.dense_packing(n=600, phi=0.55, seed=seed, relax_steps=0)
    s = make(w.params)
    s.set_state(w.pos, w.vel, w.omega, radius=w.radius)
    s.initialize_cell_distribution()
    s.set_particle_removal(False)
    s.run(1, 12)
    return w, s


def push_out(s, w, picks):
    """Move the chosen particles outside the box (CellIndex keeps their cell,
    as after a step)."""
    st = s.get_state()
    L = np.array(list(w.params.lbox))
    pos = st["pos"].copy()
    for k, i in enumerate(picks):
        pos[i, k % 3] = (0.5 + 0.01 * (k + 1)) * L[k % 3] * (1 if k % 2 == 0 else -1)
    s.update_state(pos=pos)


def picks_near_last(s, n):
    """The last particle, a particle that shares a neighbourhood with the one
    before last, and a distant one."""
    ci, _, _ = s.get_cells()
    grid = s.grid()
    pbc = [1, 1, 1]
    near = [q for q in range(n - 3) if ci[q] in neighbourhood(int(ci[n - 2]), grid, pbc)]
    return [n - 1, near[len(near) // 2], 5]


def test_removal_matches_the_restatement():
    w, o = dense_case(oracle_system)
    n = o.n
    picks = picks_near_last(o, n)
    push_out(o, w, picks)
    before = export(o)
    want = restated_removal(before, list(w.params.lbox), o.grid(), [1, 1, 1])
    assert want["moved"] > 0  # the renaming branch is exercised
    removed = o.update_particle_list()
    assert removed == 3 and o.n == n - 3
    after = export(o)
    np.testing.assert_array_equal(after["pos"], want["pos"])
    np.testing.assert_array_equal(after["vel"], want["vel"])
    np.testing.assert_array_equal(after["cell_index"], want["cell_index"])
    np.testing.assert_array_equal(after["traversal"], want["traversal"])
    np.testing.assert_array_equal(after["prev"], want["ring"])
    np.testing.assert_array_equal(after["contacts"]["imin"], want["imin"])
    np.testing.assert_array_equal(after["contacts"]["imax"], want["imax"])
    np.testing.assert_array_equal(after["contacts"]["ft"], want["ft"])
    st = o.removal_stats()
    assert st["removed"] == 3 and st["swaps"] == 2 and st["records_moved"] == want["moved"]
    # the run carries on with the smaller system
    o.run(13, 20)
    assert np.isfinite(o.get_state()["pos"]).all()


def test_run_removes_after_every_step_and_can_be_switched_off():
    w = configs.discharge(d_out=5.0, mu=0.2)
    a = oracle_system(w.params)
    b = oracle_system(w.params)
    for s in (a, b):
        s.set_state(w.pos, w.vel, w.omega, comp=w.comp)
        s.initialize_cell_distribution()
    b.set_particle_removal(False)
    a.run(1, 500)
    b.run(1, 500)
    assert a.n < w.pos.shape[0] == b.n
    assert b.escaped() > 0
    L = np.array(list(w.params.lbox))
    pa = a.get_state()["pos"]
    assert not np.any((pa > 0.5 * L) | (pa < -0.5 * L))


def test_literal_append_order_shows_the_deviation():
    """The reference appends the records particle i inherits in neighbour
    order (src/MContacts.f90:225-241); its ordered search (VerifyPairContact,
    src/MContacts.f90:329-372) then misses the later of two out-of-order
    records, and the next updating pass adds a second record for that pair.
    The oracle's literal mode does exactly that; the default mode (the one
    the GPU follows) keeps the list ordered and the history of the pair."""
    from tests.oracle_lib import load_oracle
    lib = load_oracle()
    after = {}
    for literal in (0, 1):
        w, o = dense_case(oracle_system, seed=51)
        lib.orc_set_literal_removal(o._ctx, literal)
        pos = o.get_state()["pos"].copy()
        pos[531, 0] = 0.51 * w.params.lbox[0]  # particle 531 leaves; the last one replaces it
        o.update_state(pos=pos)
        want = restated_removal(export(o), list(w.params.lbox), o.grid(), [1, 1, 1],
                                literal=bool(literal))
        assert o.update_particle_list() == 1
        ct = o.get_contacts()
        np.testing.assert_array_equal(ct["imin"], want["imin"])
        np.testing.assert_array_equal(ct["imax"], want["imax"])
        inherited = list(ct["imax"][ct["imin"] == 531])
        assert inherited == ([592, 591] if literal else [591, 592])
        o.compute_accelerations(update=True)
        ct = o.get_contacts()
        after[literal] = list(ct["imax"][ct["imin"] == 531])
    assert after[0] == [591, 592]
    assert sorted(after[1]) == [591, 591, 592]  # two records for one pair
