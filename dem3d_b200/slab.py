"""Spatial decomposition of one system into z-slabs: the host schedule.

The reference is serial; its thesis names spatial decomposition with
message passing as the way to parallelise it.  Here one large system is cut
into slabs of whole cell layers along z (cells are numbered x + Nx*(y +
Ny*z), src/MCells.f90, so a slab is a contiguous range of cells and the
sweep of src/MForces.f90:173-324 meets the slabs one after the other).  Each
slab is a context (``dem_slab_*`` in dem3d_b200.h) that holds the arrays of
every particle but advances only the particles of its layers.  The sweep's
half-shell reaches one layer up, so a MoveParticles step needs, in each of
its two force passes:

    displacement   max over slabs of the last pass's largest displacement
    RELINK         every slab
    GHOSTS         slab r+1 -> slab r   (its bottom layer)
    LOWER          slab r-1 -> slab r   (the cells of its top layer)
    TEST_PAIR      every slab
    JHALVES        slab r -> slab r+1   (results for its particles)
    FOLD           every slab
    MIGRATE_UP     slab r -> slab r+1   (particles that entered its layers)
    MIGRATE_DOWN   slab r -> slab r-1
    FINISH         every slab

With a periodic z axis the slabs form a ring; otherwise the end slabs skip
the missing neighbour.  The schedule is written once over two transports:
``LocalTransport`` (all slabs in this process: every exchange is packed on
the sending slab into its own device buffer and copied into the receiving
slab's buffer) and ``DistTransport`` (one slab per rank of a
torch.distributed group: the same buffers go by send/receive, the sizes
first).  The result is the undivided system's, bit for bit
(tests/test_gpu_slab.py).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _abi

PHASES = (_abi.SLAB_RELINK, _abi.SLAB_TEST_PAIR, _abi.SLAB_FOLD, _abi.SLAB_FINISH)
# exchange -> direction of travel (+1: to the slab above, -1: to the slab below)
DIRECTION = {_abi.SLAB_GHOSTS: -1, _abi.SLAB_LOWER: +1, _abi.SLAB_JHALVES: +1,
             _abi.SLAB_MIGRATE_UP: +1, _abi.SLAB_MIGRATE_DOWN: -1}
# (phase, exchanges that follow it) for one force pass
PASS_SCHEDULE = ((_abi.SLAB_RELINK, (_abi.SLAB_GHOSTS, _abi.SLAB_LOWER)),
                 (_abi.SLAB_TEST_PAIR, (_abi.SLAB_JHALVES,)),
                 (_abi.SLAB_FOLD, (_abi.SLAB_MIGRATE_UP, _abi.SLAB_MIGRATE_DOWN)),
                 (_abi.SLAB_FINISH, ()))


def slab_ranges(nz: int, nslabs: int):
    """Nz cell layers cut into nslabs contiguous [z0, z1) ranges of at least
    two layers each, as even as possible (the first nz % nslabs one longer)."""
    if nslabs < 1 or nz < 2 * nslabs:
        raise ValueError(f"{nz} cell layers cannot make {nslabs} slabs of two layers or more")
    base, extra = divmod(nz, nslabs)
    out, z = [], 0
    for r in range(nslabs):
        w = base + (1 if r < extra else 0)
        out.append((z, z + w))
        z += w
    return out


def neighbour(r: int, d: int, nslabs: int, periodic: bool):
    """The slab above (d = +1) or below (d = -1) slab r, or None."""
    q = r + d
    if 0 <= q < nslabs:
        return q
    return q % nslabs if periodic and nslabs > 1 else None


@dataclass
class Route:
    """One exchange of one pass as seen by slab r: whom it sends to, whom it
    receives from (None: nobody)."""
    what: int
    send_to: int | None
    recv_from: int | None


def routes(r: int, nslabs: int, periodic: bool, what: int) -> Route:
    d = DIRECTION[what]
    return Route(what, neighbour(r, d, nslabs, periodic), neighbour(r, -d, nslabs, periodic))


def global_displacement(bits) -> int:
    """The largest of the slabs' displacement bounds (FP32 bit patterns of
    non-negative floats order like the floats)."""
    return int(max(bits))


class LocalTransport:
    """All slabs in this process, on one GPU: each slab packs into its own
    device buffer, which is copied into the receiver's buffer."""

    def __init__(self, slabs, periodic: bool, cap_bytes: int):
        import torch
        self.torch = torch
        self.slabs = slabs
        self.periodic = periodic
        self.cap = int(cap_bytes)
        self.send = [torch.empty(self.cap, dtype=torch.uint8, device="cuda") for _ in slabs]
        self.recv = [torch.empty(self.cap, dtype=torch.uint8, device="cuda") for _ in slabs]
        self.bytes_moved = 0

    def displacement(self):
        bits = [s.slab_displacement() for s in self.slabs]
        g = global_displacement(bits)
        for s in self.slabs:
            s.slab_displacement(g)

    def phase(self, step, pass_, phase):
        for s in self.slabs:
            s.slab_phase(step, pass_, phase)

    def exchange(self, what):
        n = len(self.slabs)
        sizes = {}
        for r, s in enumerate(self.slabs):
            rt = routes(r, n, self.periodic, what)
            if rt.send_to is not None:
                sizes[rt.send_to] = s.slab_pack(what, self.send[r].data_ptr(), self.cap)
                src = r
                self.recv[rt.send_to][:sizes[rt.send_to]].copy_(self.send[src][:sizes[rt.send_to]])
                self.bytes_moved += sizes[rt.send_to]
        self.torch.cuda.synchronize()
        for r, s in enumerate(self.slabs):
            if r in sizes:
                s.slab_unpack(what, self.recv[r].data_ptr(), sizes[r])


class DistTransport:
    """One slab per rank of the default torch.distributed group (NCCL over
    NVLink on GPUs): every exchange is a send to one neighbour and a receive
    from the other, sizes first."""

    def __init__(self, slab, rank: int, world: int, periodic: bool, cap_bytes: int,
                 device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.slab, self.rank, self.world, self.periodic = slab, rank, world, periodic
        self.cap = int(cap_bytes)
        # the buffers live where the slab's kernels read them (a CPU device
        # only for host-side tests of the schedule with a stand-in slab)
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.send = torch.empty(self.cap, dtype=torch.uint8, device=dev)
        self.recv = torch.empty(self.cap, dtype=torch.uint8, device=dev)
        self.dev = dev
        self.bytes_moved = 0

    def displacement(self):
        t = self.torch.tensor([self.slab.slab_displacement()], dtype=self.torch.int64,
                              device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        self.slab.slab_displacement(int(t.item()))

    def phase(self, step, pass_, phase):
        self.slab.slab_phase(step, pass_, phase)

    def exchange(self, what):
        torch, dist = self.torch, self.dist
        rt = routes(self.rank, self.world, self.periodic, what)
        n_out = torch.zeros(1, dtype=torch.int64, device=self.dev)
        n_in = torch.zeros(1, dtype=torch.int64, device=self.dev)
        if rt.send_to is not None:
            n_out[0] = self.slab.slab_pack(what, self.send.data_ptr(), self.cap)
        ops = []
        if rt.send_to is not None:
            ops.append(dist.P2POp(dist.isend, n_out, rt.send_to))
        if rt.recv_from is not None:
            ops.append(dist.P2POp(dist.irecv, n_in, rt.recv_from))
        for w in dist.batch_isend_irecv(ops) if ops else []:
            w.wait()
        ops = []
        k_out, k_in = int(n_out.item()), int(n_in.item())
        if rt.send_to is not None:
            ops.append(dist.P2POp(dist.isend, self.send[:k_out], rt.send_to))
        if rt.recv_from is not None:
            ops.append(dist.P2POp(dist.irecv, self.recv[:k_in], rt.recv_from))
        for w in dist.batch_isend_irecv(ops) if ops else []:
            w.wait()
        if self.dev.type == "cuda":
            torch.cuda.synchronize()
        self.bytes_moved += k_out
        if rt.recv_from is not None:
            self.slab.slab_unpack(what, self.recv.data_ptr(), k_in)


def move_particles(transport, step: int) -> None:
    """MoveParticles(step) (src/MDEM.f90:285-369) over the slabs: the
    predictor pass with history update, then the corrector pass."""
    for pass_ in (0, 1):
        transport.displacement()
        for phase, exchanges in PASS_SCHEDULE:
            transport.phase(step, pass_, phase)
            for what in exchanges:
                transport.exchange(what)


def compose_state(slabs):
    """The state of every particle from the slab that advances it."""
    out = None
    seen = None
    for s in slabs:
        own = s.slab_owned()
        st = s.get_state()
        if out is None:
            out = {k: np.zeros_like(v) for k, v in st.items()}
            seen = np.zeros(len(own), dtype=np.int32)
        for k in st:
            out[k][own] = st[k][own]
        seen += own
    if not np.all(seen == 1):
        raise RuntimeError("a particle is advanced by no slab or by several")
    return out
