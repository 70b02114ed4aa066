"""Sharding of independent systems across ranks, on CPU with world_size-2 gloo groups:
every rank computes the same partition, the shards are disjoint and cover all systems,
the load is balanced, and per-system results gather on rank 0 over the host group."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    from faspxx_b200 import problems as P
    from faspxx_b200 import shard as S
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms, sig, _ = P.batch_systems(count=257, nrhs=1, seed=3)
    work = 5 * ms.astype(np.int64) ** 2          # ~nnz of each m x m 5-point system
    shards = S.partition(work, world)
    mine = shards[rank]
    # stand-in for the GPU solve: a per-system result that only the owner can produce
    local = {"systems": mine.tolist(), "iters": [int(m) for m in ms[mine]]}
    got = S.gather_results(dist, rank, world, local)
    if rank == 0:
        q.put((got, [s.tolist() for s in shards], S.imbalance(work, shards)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_partition_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, shards, imb = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g["systems"] for g in got] == shards
    allsys = sorted(sum(shards, []))
    assert allsys == list(range(257))
    assert imb < 1.01


def test_partition_properties():
    from faspxx_b200 import shard as S
    rng = np.random.default_rng(0)
    work = rng.integers(1, 1000, size=1000)
    for world in (1, 2, 3, 8):
        sh = S.partition(work, world)
        assert sorted(np.concatenate(sh).tolist()) == list(range(1000))
        loads = [work[s].sum() for s in sh]
        assert max(loads) - min(loads) <= work.max()
        assert S.partition(work, world)[0].tolist() == sh[0].tolist()  # deterministic
