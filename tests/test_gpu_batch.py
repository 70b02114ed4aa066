"""Batched Jacobi-PCG (fasp_gpu_batch_*): uneven shifted 2D Poisson systems with several
right-hand sides each, solved in one persistent launch, checked per system against SciPy
direct solves (solution) and the CPU oracle's CG (iteration count).

Tolerances: FP64 — relative residual <= relTol (1e-10) per right-hand side, solution within
1e-8 of the direct solve, iterations within max(2, 3%) of the oracle's CG (the batched
kernel stops on the recursive residual alone, without CG::Solve's false-convergence
recheck, so near 1e-10 the counts may differ by a couple); mixed (FP32 inner, FP64
refinement) — relative residual <= relTol (1e-8).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    from faspxx_b200 import batch as BT
    from faspxx_b200 import problems as P
    rng = np.random.default_rng(5)
    ms = rng.integers(8, 41, size=37)
    sig = rng.uniform(0.0, 1.0, size=37)
    mats = BT.shifted_poisson_batch(ms, sig)
    B = BT.Batch(mats, nrhs=4)
    b = rng.standard_normal((4, B.N))
    return B, mats, b, P


def test_batch_fp64_matches_direct_and_oracle(batch):
    import scipy.sparse.linalg as spla
    from oracle import oracle as O
    B, mats, b, P = batch
    x, it, rr, ms = B.solve(b, relTol=1e-10)
    for k, m in enumerate(mats):
        r0, r1 = int(B.sys_row[k]), int(B.sys_row[k + 1])
        S = m.scipy().tocsc()
        for j in range(4):
            bj = b[j, r0:r1]
            xs = spla.spsolve(S, bj)
            res = np.linalg.norm(bj - m.matvec(x[j, r0:r1])) / np.linalg.norm(bj)
            assert res <= 1.5e-10, (k, j, res)
            assert np.linalg.norm(x[j, r0:r1] - xs) <= 1e-8 * np.linalg.norm(xs), (k, j)
        if k % 6 == 0:  # the oracle's CG with the same stopping test, for a sample
            ref = O.solve("port", m, "cg", b[0, r0:r1], np.zeros(m.nrow), maxIter=5000,
                          minIter=0, relTol=1e-10, absTol=0.0, pcd="jacobi", pcdWeight=1.0,
                          pcdIter=1)
            assert abs(int(it[k, 0]) - ref.iters) <= max(2, 0.03 * ref.iters), \
                (k, it[k, 0], ref.iters)


def test_batch_mixed_reaches_fp64_residual(batch):
    from faspxx_b200 import capi
    B, mats, b, P = batch
    x, it, rr, ms = B.solve(b, relTol=1e-8, precision=capi.MIXED, innerRelTol=1e-4)
    assert np.all(rr <= 1e-8)
    for k, m in enumerate(mats):
        r0, r1 = int(B.sys_row[k]), int(B.sys_row[k + 1])
        for j in range(4):
            bj = b[j, r0:r1]
            res = np.linalg.norm(bj - m.matvec(x[j, r0:r1])) / np.linalg.norm(bj)
            assert res <= 1e-8, (k, j, res)


def test_batch_reliable_updates_reach_fp64_residual_in_fp64_iterations(batch):
    """FP32 iterations with block-local FP64 reliable updates: every system and right-hand
    side reaches the FP64 relative residual 1e-8, in the FP64 iteration count (+5% +2)."""
    from faspxx_b200 import capi
    B, mats, b, P = batch
    x64, it64, _, _ = B.solve(b, relTol=1e-8, precision=capi.FP64)
    x, it, rr, ms = B.solve(b, relTol=1e-8, precision=capi.MIXED_RELIABLE, innerRelTol=1e-2)
    assert np.all(rr <= 1e-8)
    for k, m in enumerate(mats):
        r0, r1 = int(B.sys_row[k]), int(B.sys_row[k + 1])
        for j in range(4):
            bj = b[j, r0:r1]
            res = np.linalg.norm(bj - m.matvec(x[j, r0:r1])) / np.linalg.norm(bj)
            assert res <= 1e-8, (k, j, res)
    assert it.sum() <= it64.sum() * 1.05 + 2 * it.size
    x2 = B.solve(b, relTol=1e-8, precision=capi.MIXED_RELIABLE, innerRelTol=1e-2)[0]
    assert np.array_equal(x, x2)


def test_batch_autotune_and_repeatability(batch):
    B, mats, b, P = batch
    shape, ms = B.autotune(b)
    x1 = B.solve(b, relTol=1e-10)[0]
    x2 = B.solve(b, relTol=1e-10)[0]
    assert np.array_equal(x1, x2)  # block-local fixed-order reductions: deterministic
    assert shape in [(128, 8), (128, 16), (256, 4), (256, 8), (512, 2), (512, 4)]


def test_batch_rejects_coupled_systems():
    from faspxx_b200 import batch as BT
    from faspxx_b200 import capi
    from faspxx_b200 import problems as P
    mats = [P.poisson2d(4), P.poisson2d(4)]
    sys_row, A = BT.block_diagonal(mats)
    A.colInd[0] = 20  # row 0 of system 0 reaching into system 1
    import ctypes as C
    capi.init(0)
    d = [BT._Dev(a) for a in (sys_row, A.rowPtr, A.colInd, A.values)]
    h = C.c_void_p()
    code = capi.lib.fasp_gpu_batch_create(2, d[0].p, A.nnz, d[1].p, d[2].p, d[3].p, 1,
                                          C.byref(h))
    assert code == -17
