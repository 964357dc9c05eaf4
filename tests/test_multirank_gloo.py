"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the timed
region is the max over ranks, the value aggregates every rank's system,
every rank of the 1M-sphere workload advances a different member (seed +
rank), and the ensemble workload's systems are split between the ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = 100.0 + 50.0 * rank
    mx = bench.reduce_max(ms, world, device="cpu")
    v = bench.aggregate_rate(1000, world, 10, mx)
    from dem3d_b200 import configs
    w = configs.dense_packing(n=512, phi=0.5, seed=bench.rank_seed(1001, rank), relax_steps=0)
    q.put((rank, mx, v, float(w.vel[0, 0])))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(world))
    assert all(r[1] == 150.0 for r in res)                  # max over ranks
    assert all(abs(r[2] - 1000 * 2 * 10 / 0.150) < 1e-6 for r in res)
    assert res[0][3] != res[1][3]                            # distinct members


def _shard_worker(rank, world, port, q):
    import numpy as np
    import torch
    import torch.distributed as dist

    from dem3d_b200 import configs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    e = configs.settling_ensemble(n_systems=37, seed=1003, nmin=50, nmax=400)
    mine = e.shard(rank, world)
    # every rank's systems are the ensemble's systems, unchanged
    for j, k in enumerate(mine.info["systems"]):
        a, b = mine.system(j), e.system(k)
        for x, y in zip(a[1:], b[1:]):
            assert np.array_equal(x, y)
        assert a[0].lbox[2] == b[0].lbox[2]
    counts = torch.tensor([mine.n, len(mine.counts)], dtype=torch.int64)
    dist.all_reduce(counts)
    ids = [None] * world
    dist.all_gather_object(ids, mine.info["systems"])
    q.put((rank, int(counts[0]), int(counts[1]), sorted(sum(ids, [])), mine.n, e.n))
    dist.barrier()
    dist.destroy_process_group()


def test_ensemble_systems_sharded_over_ranks():
    """bench.py's ensemble workload on several ranks: the systems are split
    between the ranks (every world-th system), each exactly once, and the
    particle counts of the ranks are balanced."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(world))
    total = res[0][5]
    for r in res:
        assert r[1] == total and r[2] == 37          # every particle and system once
        assert r[3] == list(range(37))
    share = [r[4] / total for r in res]
    assert all(0.3 < x < 0.7 for x in share), share
