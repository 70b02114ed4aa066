"""16-bit column offsets of the CSR form (fasp_gpu_mat_set_col16): the thread-per-row kernels
read colInd[k] - row as int16 instead of the 32-bit colInd when every entry lies within
32,767 columns of its row. The entries and their order are the same, so every result must be
bit-identical with the offsets on and off: MAT::Apply and MAT::Residual, FP64 CG, BiCGStab
and GMRES solves and the FP32-iteration CG (iterations, x and history), on the bundled and
synthetic matrices in their CSR form; the offsets are built for transposes too, and not
built when an entry lies farther from its row."""
import numpy as np
import pytest

from tests.golden import cases as G

pytestmark = pytest.mark.gpu

MATS = ["fdm_10X10", "fem_small", "poisson3d_12", "convdiff_pe10", "vardiff_8"]


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return capi, sol


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("name", MATS)
def test_apply_and_residual_bit_identical(gpu, name):
    capi, sol = gpu
    A = G.matrix(name)
    M = sol.MAT(A)
    M.SetRowClass(0)
    M.SetLanes(1)
    assert M.Col16Info() == (True, False)  # built, off by default
    rng = np.random.default_rng(3)
    x, b = sol.DVec.from_numpy(rng.standard_normal(A.mcol)), sol.DVec.from_numpy(
        rng.standard_normal(A.nrow))
    out = []
    for on in (True, False):
        M.SetCol16(on)
        assert M.Col16Info()[1] == on
        y, r = sol.DVec(A.nrow), sol.DVec(A.nrow)
        M.Apply(x, y)
        M.Residual(b, x, r)
        out.append((y.numpy(), r.numpy()))
    assert np.array_equal(_bits(out[0][0]), _bits(out[1][0]))
    assert np.array_equal(_bits(out[0][1]), _bits(out[1][1]))


@pytest.mark.parametrize("alg", ["cg", "bicgstab", "gmres", "cg_mixed"])
@pytest.mark.parametrize("name", ["poisson3d_12", "vardiff_8", "convdiff_pe10"])
def test_solves_bit_identical(gpu, name, alg):
    capi, sol = gpu
    if alg.startswith("cg") and name == "convdiff_pe10":
        pytest.skip("CG needs a symmetric matrix")
    A = G.matrix(name)
    b = A.matvec(np.random.default_rng(5).uniform(-1, 1, A.nrow))
    kw = dict(maxIter=500, minIter=0, relTol=1e-10, absTol=0.0, pcd="jacobi",
              pcdWeight=2.0 / 3.0 if alg != "cg" and alg != "cg_mixed" else 1.0, pcdIter=1)
    if alg == "gmres":
        kw.update(restart=30, maxRestart=30, minRestart=30)
    out = []
    for on in (True, False):
        M = sol.MAT(A)
        M.SetRowClass(0)
        M.SetLanes(1)
        M.SetCol16(on)
        s = sol.configure("cg" if alg == "cg_mixed" else alg, **kw)
        if alg == "cg_mixed":
            s.SetPrecision(capi.MIXED_RELIABLE)
        s.Setup(M)
        x = np.zeros(A.nrow)
        code = s.Solve(b, x)
        out.append((code, s.GetIterations(), x, s.History()))
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert np.array_equal(_bits(out[0][2]), _bits(out[1][2]))
    assert np.array_equal(out[0][3], out[1][3], equal_nan=True)


def test_transpose_gets_offsets_and_far_entries_do_not(gpu):
    capi, sol = gpu
    from faspxx_b200 import problems as P
    A = G.matrix("convdiff_pe10")
    assert sol.MAT(A).Transpose().Col16Info()[0]
    n = 40000  # one entry 39,999 columns from its row
    rp = np.arange(n + 1, dtype=np.uint32)
    ci = np.arange(n, dtype=np.uint32)
    rp2 = np.concatenate([[0], np.arange(2, n + 2, dtype=np.uint32)])
    ci2 = np.concatenate([[0, n - 1], ci[1:]]).astype(np.uint32)
    va2 = np.ones(n + 1)
    far = sol.MAT(P.CSRMatrix(n, n, rp2, ci2, va2))
    assert far.Col16Info() == (False, False)
    near = sol.MAT(P.CSRMatrix(n, n, rp, ci, np.ones(n)))
    assert near.Col16Info()[0]
