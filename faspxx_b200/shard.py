"""Multi-GPU sharding of independent systems: one process per GPU, no data-path collective.

Batched solves partition naturally: each system is independent, so every rank takes a
share of the systems (greedy longest-processing-time by nnz, deterministic, the same on
every rank), solves it on its own GPU with the batched kernel, and only the per-system
results (iteration counts, residuals) travel to rank 0 over the host process group. A
single large system does not shard here: the benchmark runs replicas of it instead.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(work: np.ndarray, world: int) -> list[np.ndarray]:
    """Split item indices into `world` shards with near-equal total work (LPT greedy:
    largest item to the currently lightest shard; ties broken by shard number)."""
    work = np.asarray(work, dtype=np.int64)
    order = np.argsort(-work, kind="stable")
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(int(i))
        heapq.heappush(heap, (load + int(work[i]), r))
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def imbalance(work: np.ndarray, shards: list[np.ndarray]) -> float:
    """max shard load / mean shard load."""
    loads = np.array([np.asarray(work)[s].sum() for s in shards], dtype=np.float64)
    return float(loads.max() / max(loads.mean(), 1.0))


def gather_results(dist, rank: int, world: int, local: dict):
    """Host-side gather of per-system results to rank 0 (None elsewhere)."""
    if dist is None or world == 1:
        return [local]
    out = [None] * world if rank == 0 else None
    dist.gather_object(local, out, dst=0)
    return out


def solve_shard(mats, rhs, shard, relTol=1e-8, precision=0):
    """Solve this rank's systems with one batched launch on the current GPU."""
    from .batch import Batch
    sub = [mats[i] for i in shard]
    B = Batch(sub, nrhs=rhs[shard[0]].shape[0])
    b = np.zeros((B.nrhs, B.N))
    for k, i in enumerate(shard):
        b[:, B.sys_row[k]:B.sys_row[k + 1]] = rhs[i]
    x, it, rr, ms = B.solve(b, relTol=relTol, precision=precision)
    return {"systems": shard.tolist(), "iters": it.tolist(), "resRel": rr.max(axis=1).tolist(),
            "ms": ms}
