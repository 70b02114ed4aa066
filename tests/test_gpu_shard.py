"""Sharding of the batched workload on one GPU: the systems split into two shards
(shard.partition, LPT by nnz) and solved shard after shard with the batched kernel give,
system by system, the same iteration counts and final residuals as one unsharded launch --
bit for bit, because each system is solved by one thread block in a fixed order whatever
else shares the launch. So the per-rank results that bench.py --workload batch gathers under
torchrun are the unsharded batch's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_two_shards_equal_the_unsharded_batch():
    from faspxx_b200 import capi, problems as P, shard as S
    capi.init(0)
    ms, sig, rhs = P.batch_systems(count=96, mlo=8, mhi=48, nrhs=2, seed=5)
    mats = [P.poisson2d(int(m), shift=float(s)) for m, s in zip(ms, sig)]
    full = S.solve_shard(mats, rhs, np.arange(len(mats)))
    shards = S.partition(5 * ms.astype(np.int64) ** 2, 2)
    assert sorted(np.concatenate(shards).tolist()) == list(range(len(mats)))
    got_it, got_rr = {}, {}
    for sh in shards:
        r = S.solve_shard(mats, rhs, sh)
        for k, sysid in enumerate(r["systems"]):
            got_it[sysid] = r["iters"][k]
            got_rr[sysid] = r["resRel"][k]
    for k in range(len(mats)):
        assert got_it[k] == full["iters"][k], k
        assert got_rr[k] == full["resRel"][k], k
