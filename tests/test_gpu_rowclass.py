"""Compressed forms of constant-coefficient matrices in the thread-per-row SpMV kernels:
row classes (a 2-byte class id per row into a table of (column offset, value) lists) and
stencil masks (a 16-bit mask per row over one sorted offset list passed as kernel
parameters).

Bar: bit-exact. All three forms (CSR, classes, masks) accumulate each row's entries in CSR
order with one FMA per entry, so MAT::Apply, MAT::Residual and whole solves (iteration
counts, solutions and residual histories) are identical whichever form is in use. One
exception: the FP32 iterations of mixed-precision CG on stencil masks with n % 4 == 0 run
four rows per thread (the same bits per row, another grid and order of the FP32 partial
sums), so there the masks form is held to the outcome of the other two.
"""
import numpy as np
import pytest

from faspxx_b200 import problems as P
from tests.golden import cases as G

pytestmark = pytest.mark.gpu

CSR, CLASSES, MASKS = 0, 1, 2


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


def _stencils():
    return {
        "poisson2d_40": (P.poisson2d(40), 5),
        "poisson3d_20": (P.poisson3d(20), 7),
        "convdiff3d_16_pe10": (P.convdiff3d(16, 10.0), 7),
        "fdm_10X10": (G.matrix("fdm_10X10"), None),
    }


@pytest.mark.parametrize("name", list(_stencils()))
def test_apply_and_residual_bit_exact(gpu, name):
    A, stencil = _stencils()[name]
    M = gpu.MAT(A)
    mode, classes, entries, st = M.RowClassInfo()
    assert 0 < classes <= 4096 and entries <= max(64, A.nnz // 8)
    if stencil is not None:
        assert mode == MASKS and st == stencil
    rng = np.random.default_rng(1)
    x = gpu.DVec.from_numpy(rng.standard_normal(A.mcol))
    b = gpu.DVec.from_numpy(rng.standard_normal(A.nrow))
    out = {}
    for form in (MASKS, CLASSES, CSR):
        M.SetRowClass(form)
        y, r = gpu.DVec(A.nrow), gpu.DVec(A.nrow)
        M.Apply(x, y)
        M.Residual(b, x, r)
        out[form] = (y.numpy(), r.numpy())
    assert M.RowClassInfo()[0] == CSR
    for form in (MASKS, CLASSES):
        assert np.array_equal(out[form][0], out[CSR][0]), form
        assert np.array_equal(out[form][1], out[CSR][1]), form
    ref = A.matvec(x.numpy())
    assert np.max(np.abs(out[CSR][0] - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_variable_coefficients_stay_csr(gpu):
    kappa = 10.0 ** np.random.default_rng(2).uniform(-1, 1, 12 ** 3)
    M = gpu.MAT(P.vardiff3d(12, kappa))
    assert M.RowClassInfo() == (CSR, 0, 0, 0)
    M.SetRowClass(MASKS)  # nothing to switch on
    assert M.RowClassInfo()[0] == CSR


def test_classes_without_a_common_stencil(gpu):
    """A Neumann-like boundary (diagonal differs on boundary rows) has few classes but no
    single value per offset: classes are built, masks are not."""
    A = P.poisson2d(30)
    vals = A.values.copy()
    diag = np.array([A.rowPtr[i] + np.nonzero(A.colInd[A.rowPtr[i]:A.rowPtr[i + 1]] == i)[0][0]
                     for i in range(A.nrow)])
    cnt = np.diff(A.rowPtr.astype(np.int64))
    vals[diag] = cnt - 1.0  # diagonal = number of neighbours
    B = P.CSRMatrix(A.nrow, A.mcol, A.rowPtr, A.colInd, vals)
    M = gpu.MAT(B)
    mode, classes, _, st = M.RowClassInfo()
    assert mode == CLASSES and classes > 1 and st == 0
    x = gpu.DVec.from_numpy(np.random.default_rng(3).standard_normal(B.nrow))
    y1, y0 = gpu.DVec(B.nrow), gpu.DVec(B.nrow)
    M.Apply(x, y1)
    M.SetRowClass(CSR)
    M.Apply(x, y0)
    assert np.array_equal(y1.numpy(), y0.numpy())


# 81^3 = 531,441 rows: more than the resident grid's threads, so the FP32 CG kernel on the
# CSR form takes rows two per thread (and one row on the threads past the last pair)
@pytest.mark.parametrize("alg,prec,dim", [("cg", "FP64", 18), ("cg", "MIXED_RELIABLE", 17),
                                          ("cg", "MIXED_RELIABLE", 18),
                                          ("cg", "MIXED_RELIABLE", 81),
                                          ("bicgstab", "FP64", 14), ("gmres", "FP64", 14),
                                          ("gmres", "MIXED", 14), ("gmres_left", "FP64", 14),
                                          ("fgmres", "MIXED", 14)])
def test_solves_identical_in_every_form(gpu, alg, prec, dim):
    from faspxx_b200 import capi
    A = P.convdiff3d(dim, 0.1) if alg != "cg" else P.poisson3d(dim)
    b = A.matvec(np.random.default_rng(4).uniform(-1, 1, A.nrow))
    out = []
    for form in (CSR, CLASSES, MASKS):
        M = gpu.MAT(A)
        M.SetRowClass(form)
        s = gpu.configure(alg, maxIter=2000, relTol=1e-9, absTol=0.0, pcd="jacobi",
                          pcdWeight=2.0 / 3.0 if alg != "cg" else 1.0, pcdIter=1)
        if prec != "FP64":
            s.SetPrecision(getattr(capi, prec))
        s.Setup(M)
        x = np.zeros(A.nrow)
        code = s.Solve(b, x)
        out.append((code, s.GetIterations(), x, np.nan_to_num(s.History())))
    four_rows = alg == "cg" and prec != "FP64" and A.nrow % 4 == 0
    for o in out[1:] if not four_rows else out[1:2]:
        assert o[0] == out[0][0] == 0 and o[1] == out[0][1]
        assert np.array_equal(o[2], out[0][2])
        assert np.array_equal(o[3], out[0][3])
    if four_rows:
        code, its, x, hist = out[2]
        assert code == 0 and abs(its - out[0][1]) <= 1
        assert np.linalg.norm(x - out[0][2]) <= 1e-6 * np.linalg.norm(out[0][2])
        k = min(len(hist), len(out[0][3])) - 2
        np.testing.assert_allclose(hist[:k], out[0][3][:k], rtol=1e-2, atol=0.0)


def _banded(shape, offsets, vals):
    return P._from_stencil(shape, offsets, lambda k: vals[k])


@pytest.mark.parametrize("name", ["band3", "band27", "grid18", "grid32"])
def test_four_row_path_every_offset_kind(gpu, name):
    """Mixed-precision CG on stencil masks with n % 4 == 0 runs four rows per thread. Its
    three ways of reaching a neighbour -- an aligned 16-byte group (d % 4 == 0), warp
    shuffles of the neighbouring lanes' groups (|d| < 4) and two aligned groups (the rest)
    -- and the seven-point kernel that walks columns of planes (plane stride a multiple of
    128, grid32) must give the solve of the row-per-thread kernel on the CSR form."""
    from faspxx_b200 import capi
    if name == "band3":      # offsets -3 .. 3: shuffles reaching three elements each way
        A = _banded((1000, 1, 1), [(d, 0, 0) for d in range(-3, 4)],
                    [-0.1, -0.2, -0.5, 2.0, -0.5, -0.2, -0.1])
    elif name == "band27":   # offsets +-2 (shuffles) and +-7 (two groups)
        A = _banded((1000, 1, 1), [(-7, 0, 0), (-2, 0, 0), (0, 0, 0), (2, 0, 0), (7, 0, 0)],
                    [-0.4, -0.55, 2.0, -0.55, -0.4])
    elif name == "grid18":   # 18 x 10 x 8 grid: +-1 shuffles, +-18 two groups, +-180 aligned
        A = _banded((18, 10, 8), P._OFF3D, [-1.0, -1.0, -1.0, 6.0, -1.0, -1.0, -1.0])
    else:                    # 32 x 32 x 12 grid: planes of 1024 rows walked in columns
        A = _banded((32, 32, 12), P._OFF3D, [-1.0, -1.0, -1.0, 6.0, -1.0, -1.0, -1.0])
    assert A.nrow % 4 == 0
    b = A.matvec(np.random.default_rng(7).uniform(-1, 1, A.nrow))
    out = []
    for form in (CSR, MASKS):
        M = gpu.MAT(A)
        M.SetRowClass(form)
        s = gpu.configure("cg", maxIter=3000, relTol=1e-9, absTol=0.0, pcd="jacobi",
                          pcdWeight=1.0, pcdIter=1)
        s.SetPrecision(capi.MIXED_RELIABLE)
        s.Setup(M)
        x = np.zeros(A.nrow)
        code = s.Solve(b, x)
        out.append((code, s.GetIterations(), x))
    assert out[0][0] == out[1][0] == 0
    assert abs(out[0][1] - out[1][1]) <= 1
    assert np.linalg.norm(out[1][2] - out[0][2]) <= 1e-6 * np.linalg.norm(out[0][2])
    r = b - A.matvec(out[1][2])
    assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("shape", [(32, 32, 12), (20, 20, 10), (40, 40)])
def test_fp64_two_row_path(gpu, oracle_built, shape):
    """FP64 CG on 5- and 7-point stencil masks with n % 2 == 0 runs two rows per thread
    (walking columns of planes when the plane stride is a multiple of 64: 32 x 32 x 12).
    Every row is formed as in the row-per-thread kernel; only the grouping of the FP64 dot
    products differs, so the solve must agree with the CSR form and with the oracle's
    iteration count."""
    O = oracle_built
    if len(shape) == 3:
        A = _banded(shape, P._OFF3D, [-1.0, -1.0, -1.0, 6.0, -1.0, -1.0, -1.0])
    else:
        A = _banded((shape[0], shape[1], 1), P._OFF2D, [-1.0, -1.0, 4.0, -1.0, -1.0])
    b = A.matvec(np.random.default_rng(11).uniform(-1, 1, A.nrow))
    kw = dict(maxIter=3000, relTol=1e-10, absTol=0.0, pcd="jacobi", pcdWeight=1.0, pcdIter=1)
    out = []
    for form in (CSR, MASKS):
        M = gpu.MAT(A)
        M.SetRowClass(form)
        s = gpu.configure("cg", **kw)
        s.Setup(M)
        x = np.zeros(A.nrow)
        code = s.Solve(b, x)
        out.append((code, s.GetIterations(), x, np.nan_to_num(s.History())))
    ref = O.solve("port", A, "cg", b, np.zeros(A.nrow), **kw)
    assert out[0][0] == out[1][0] == ref.code == 0
    assert out[0][1] == out[1][1]
    assert abs(out[1][1] - ref.iters) <= 1
    assert np.linalg.norm(out[1][2] - out[0][2]) <= 1e-9 * np.linalg.norm(out[0][2])
    assert np.linalg.norm(out[1][2] - ref.x) <= 1e-8 * np.linalg.norm(ref.x)
    np.testing.assert_allclose(out[1][3], out[0][3], rtol=1e-6, atol=0.0)


def test_mixed_cg_irregular_csr_rows(gpu):
    """FP32 CG iterations on a general CSR matrix of 400,001 rows with 1 to about 30 entries
    a row, and rows 0 and n-1 (where the clipped columns pile up) with a few thousand (more
    rows than the resident grid's threads: two rows per thread, rows of unequal length side
    by side, one row on the threads past the last pair). The mixed solve must
    meet the FP64 tolerance and agree with the FP64 solve, whose kernel walks one row at a
    time."""
    import scipy.sparse as sp
    from faspxx_b200 import capi
    n = 400_001
    rng = np.random.default_rng(5)
    deg = rng.integers(0, 8, n)
    rows = np.repeat(np.arange(n), deg)
    cols = np.clip(rows + rng.integers(-5000, 5001, rows.size), 0, n - 1)
    keep = rows != cols
    S = sp.coo_matrix((-rng.uniform(0.1, 1.0, keep.sum()), (rows[keep], cols[keep])),
                      shape=(n, n)).tocsr()
    S = (S + S.T).tocsr()
    S.sum_duplicates()
    d = -np.asarray(S.sum(axis=1)).ravel() + rng.uniform(0.05, 0.5, n)
    S = (S + sp.diags(d)).tocsr()
    S.sort_indices()
    cnt = np.diff(S.indptr)
    assert cnt.min() == 1 and cnt[1:-1].max() >= 20 and min(cnt[0], cnt[-1]) > 1000
    A = P.CSRMatrix(n, n, S.indptr.astype(np.uint32), S.indices.astype(np.uint32),
                    S.data.astype(np.float64))
    b = A.matvec(rng.uniform(-1, 1, n))
    out = {}
    for prec in ("FP64", "MIXED_RELIABLE"):
        M = gpu.MAT(A)
        assert M.RowClassInfo()[0] == CSR
        s = gpu.configure("cg", maxIter=2000, relTol=1e-9, absTol=0.0, pcd="jacobi",
                          pcdWeight=1.0, pcdIter=1)
        s.SetPrecision(getattr(capi, prec))
        s.Setup(M)
        x = np.zeros(n)
        assert s.Solve(b, x) == 0
        assert np.linalg.norm(b - A.matvec(x)) <= 1e-9 * np.linalg.norm(b)
        out[prec] = (s.GetIterations(), x)
    assert abs(out["MIXED_RELIABLE"][0] - out["FP64"][0]) <= max(3, out["FP64"][0] // 20)
    assert np.linalg.norm(out["MIXED_RELIABLE"][1] - out["FP64"][1]) <= \
        1e-7 * np.linalg.norm(out["FP64"][1])
