"""The slab decomposition's host schedule over torch.distributed (gloo, on
CPU, world sizes 2 and 3): dem3d_b200.slab's DistTransport and
move_particles drive a stand-in slab that follows a known motion of
particles between cell layers.  Every exchange must reach the right
neighbour with the right content: the ghost layer is the slab above's
bottom layer, the lower cells are the slab below's top layer, the results
for ghosts go back to their owner, leavers reach the slab they entered, and
every particle is owned by exactly one slab after every pass."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dem3d_b200 import _abi
from dem3d_b200 import slab as S


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class ToySlab:
    """Particles on cell layers: after pass k, particle i sits on layer
    (z0[i] + k * dir[i]) mod nz (at most one layer per pass, the bound the
    real slabs rely on).  The slab owns the particles on its layers and
    checks every buffer it receives against that known motion."""

    def __init__(self, r, ranges, nz, n=400, periodic=True, seed=3):
        rng = np.random.default_rng(seed)
        self.r, self.ranges, self.nz, self.periodic = r, ranges, nz, periodic
        self.z0, self.z1 = ranges[r]
        self.start = rng.integers(0, nz, n)
        self.dir = rng.integers(-1, 2, n) if periodic else np.zeros(n, dtype=np.int64)
        self.k = 0                      # passes completed
        self.owned = self._truth_owned(0)
        self.ghosts = None
        self.received = []
        self.errors = []

    def layer(self, k):
        return (self.start + k * self.dir) % self.nz

    def _truth_owned(self, k):
        z = self.layer(k)
        return (z >= self.z0) & (z < self.z1)

    # the dem_slab_* surface
    def slab_displacement(self, set_bits=None):
        mine = 1000 + 7 * self.r + self.k
        if set_bits is not None and set_bits != 1000 + 7 * (len(self.ranges) - 1) + self.k:
            self.errors.append(("displacement", set_bits))
        return mine

    def slab_phase(self, step, pass_, phase):
        if phase == _abi.SLAB_FOLD:
            self.next = self.layer(self.k + 1)
        if phase == _abi.SLAB_FINISH:
            self.k += 1
            want = self._truth_owned(self.k)
            if not np.array_equal(self.owned, want):
                self.errors.append(("owned", self.k, int(np.count_nonzero(self.owned != want))))

    def _write(self, ptr, cap, arr):
        b = np.asarray(arr, dtype=np.int32).tobytes()
        assert len(b) + 8 <= cap
        head = np.array([len(b) // 4, self.r], dtype=np.int32).tobytes()
        ctypes.memmove(ptr, head + b, len(head) + len(b))
        return len(head) + len(b)

    def _read(self, ptr, nbytes):
        raw = ctypes.string_at(ptr, nbytes)
        h = np.frombuffer(raw[:8], dtype=np.int32)
        return int(h[1]), np.frombuffer(raw[8:8 + 4 * int(h[0])], dtype=np.int32)

    def _layer_ids(self, z):
        return np.flatnonzero(self.owned & (self.layer(self.k) == z % self.nz))

    def slab_pack(self, what, ptr, cap):
        if what == _abi.SLAB_GHOSTS:
            return self._write(ptr, cap, self._layer_ids(self.z0))
        if what == _abi.SLAB_LOWER:
            return self._write(ptr, cap, self._layer_ids(self.z1 - 1))
        if what == _abi.SLAB_JHALVES:
            return self._write(ptr, cap, self.ghosts)
        up = what == _abi.SLAB_MIGRATE_UP
        target = (self.z1 if up else self.z0 - 1) % self.nz
        leave = np.flatnonzero(self.owned & (self.next == target))
        self.owned[leave] = False
        return self._write(ptr, cap, leave)

    def slab_unpack(self, what, ptr, nbytes):
        src, ids = self._read(ptr, nbytes)
        self.received.append((what, src))
        z = self.layer(self.k)
        if what == _abi.SLAB_GHOSTS:
            want = np.flatnonzero(z == self.z1 % self.nz)
            if not np.array_equal(np.sort(ids), want):
                self.errors.append(("ghosts", self.k))
            self.ghosts = ids.copy()
        elif what == _abi.SLAB_LOWER:
            want = np.flatnonzero(z == (self.z0 - 1) % self.nz)
            if not np.array_equal(np.sort(ids), want):
                self.errors.append(("lower", self.k))
        elif what == _abi.SLAB_JHALVES:
            want = np.flatnonzero(z == self.z0)
            if not np.array_equal(np.sort(ids), want):
                self.errors.append(("jhalves", self.k))
        else:
            nxt = self.layer(self.k + 1)
            if not np.all((nxt[ids] >= self.z0) & (nxt[ids] < self.z1)):
                self.errors.append(("migrants", self.k))
            if np.any(self.owned[ids]):
                self.errors.append(("owned twice", self.k))
            self.owned[ids] = True


def _worker(rank, world, port, periodic, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    nz = 3 * world + 1
    ranges = S.slab_ranges(nz, world)
    slab = ToySlab(rank, ranges, nz, periodic=periodic)
    tr = S.DistTransport(slab, rank, world, periodic, 1 << 16, device=torch.device("cpu"))
    for step in range(4, 10):
        S.move_particles(tr, step)
    owned = torch.tensor(slab.owned.astype(np.int32))
    everyone = [torch.zeros_like(owned) for _ in range(world)]
    dist.all_gather(everyone, owned)
    counts = sum(t.numpy() for t in everyone)
    q.put((rank, slab.errors, [tuple(x) for x in slab.received[:5]], counts.min(), counts.max(),
           tr.bytes_moved))
    dist.barrier()
    dist.destroy_process_group()


def test_slab_ranges_and_routes():
    assert S.slab_ranges(7, 3) == [(0, 3), (3, 5), (5, 7)]
    with pytest.raises(ValueError):
        S.slab_ranges(5, 3)
    # a ring when z is periodic, a chain otherwise
    assert S.routes(0, 3, True, _abi.SLAB_GHOSTS) == S.Route(_abi.SLAB_GHOSTS, 2, 1)
    assert S.routes(0, 3, False, _abi.SLAB_GHOSTS) == S.Route(_abi.SLAB_GHOSTS, None, 1)
    assert S.routes(2, 3, False, _abi.SLAB_JHALVES) == S.Route(_abi.SLAB_JHALVES, None, 1)
    assert S.global_displacement([3, 9, 4]) == 9


@pytest.mark.parametrize("world,periodic", [(2, True), (3, True), (3, False)])
def test_slab_schedule_over_gloo(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, periodic, q))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(world))
    for rank, errors, received, cmin, cmax, moved in res:
        assert errors == [], (rank, errors)
        assert cmin == 1 and cmax == 1      # every particle owned exactly once
        assert moved > 0
        if periodic:
            # the first exchanges: ghosts from the slab above, cells from below
            assert received[0] == (_abi.SLAB_GHOSTS, (rank + 1) % world)
            assert received[1] == (_abi.SLAB_LOWER, (rank - 1) % world)
