"""ReadMat's conversions on the GPU (fasp_gpu_mat_create_coo, fasp_gpu_mat_create_csr_raw).

Parity bar: bit-exact. The row pointers, column indices and values of the built matrix
equal the reference's MTXtoMAT / SortCSRRow + CSRtoMAT results (tests/golden/
reference_ingest.*, written from the compiled reference) on the bundled data files and on
synthetic inputs with shuffled entries, duplicates, missing diagonals and long rows; at
sizes beyond the fixtures they equal the oracle's restatement (pinned on the same
fixtures) and, for shuffled stencil matrices, the stencil's own sorted CSR. Where the
reference leaves the MAT empty and returns SUCCESS (a column out of range, a row >= mcol
without a diagonal), the GPU returns ERROR_MAT_DATA (-17).
"""
import ctypes as C

import numpy as np
import pytest

from faspxx_b200 import problems as P
from tests.golden import cases as G

pytestmark = pytest.mark.gpu

CASES = G.ingest_cases()


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    return oracle


def _build(gpu, kind, nrow, mcol, a, b, v):
    if kind == "mtx":
        return gpu.MAT.FromCOO(nrow, mcol, a, b, v)
    return gpu.MAT.FromCSRRaw(nrow, a, b, v, mcol=mcol)


def _diag_ptr(rp, ci):
    """FormDiagPtr (MAT.cxx:917-928): the first entry of each row on the diagonal."""
    out = np.zeros(len(rp) - 1, np.uint32)
    for i in range(len(rp) - 1):
        hit = np.nonzero(ci[rp[i]:rp[i + 1]] == i)[0]
        out[i] = rp[i] + hit[0] if len(hit) else 0
    return out


def _same(M, expected):
    A = M.download()
    for got, want in zip((A.rowPtr, A.colInd, A.values), expected):
        assert got.dtype == want.dtype and np.array_equal(got, want)


@pytest.mark.parametrize("name", sorted(CASES))
def test_matches_reference_readmat(gpu, name):
    from faspxx_b200 import capi
    c = CASES[name]
    if c["expected"] is None:
        with pytest.raises(capi.FaspError) as e:
            _build(gpu, c["kind"], c["nrow"], c["mcol"], *c["inputs"])
        assert e.value.code == -17
        return
    M = _build(gpu, c["kind"], c["nrow"], c["mcol"], *c["inputs"])
    assert (M.GetRowSize(), M.GetColSize(), M.GetNNZ()) == (c["nrow"], c["mcol"], c["nnz"])
    _same(M, c["expected"])
    if c["nrow"] == c["mcol"]:
        assert np.array_equal(M.diag_ptr(), _diag_ptr(*c["expected"][:2]))


class _Dev:
    """A device copy of a host array (the ``ptr``/``n`` interface the constructors read)."""

    def __init__(self, a):
        from faspxx_b200 import capi
        self.a = np.ascontiguousarray(a)
        self.n = len(self.a)
        self.ptr = C.c_void_p()
        capi.check(capi.lib.fasp_gpu_malloc(C.byref(self.ptr), max(16, self.a.nbytes)), "malloc")
        capi.check(capi.lib.fasp_gpu_memcpy_h2d(self.ptr, self.a.ctypes.data, self.a.nbytes),
                   "h2d")

    def __del__(self):
        from faspxx_b200 import capi
        capi.lib.fasp_gpu_free(self.ptr)


@pytest.mark.parametrize("name", ["nos7_mtx", "fem_small_csr", "long_rows_mtx"])
def test_device_arrays(gpu, name):
    c = CASES[name]
    a, b, v = c["inputs"]
    M = _build(gpu, c["kind"], c["nrow"], c["mcol"], _Dev(a.astype(np.uint32)),
               _Dev(b.astype(np.uint32)), _Dev(v.astype(np.float64)))
    _same(M, c["expected"])


@pytest.mark.parametrize("name,ext", [("nos7_mtx", "mtx"), ("fem_small_csr", "csr"),
                                      ("random_dup_mtx", "mtx"), ("dup1_csr", "csr")])
def test_readmat_files(gpu, tmp_path, name, ext):
    c = CASES[name]
    p = str(tmp_path / f"A.{ext}")
    if ext == "mtx":
        G.write_mtx(p, c["nrow"], c["mcol"], *c["inputs"])
    else:
        G.write_csr(p, c["nrow"], *c["inputs"])
    _same(gpu.ReadMat(p), c["expected"])


def test_readmat_unknown_extension(gpu):
    from faspxx_b200 import capi
    with pytest.raises(capi.FaspError) as e:
        gpu.ReadMat("matrix.txt")
    assert e.value.code == -11


def _random_coo(rng, nrow, mcol, per_row):
    k = rng.integers(0, per_row + 1, size=nrow)
    ri = np.repeat(np.arange(nrow, dtype=np.int64), k)
    ci = rng.integers(0, mcol, size=len(ri))
    dup = rng.random(len(ri)) < 0.05
    ri, ci = np.concatenate([ri, ri[dup]]), np.concatenate([ci, ci[dup]])
    va = rng.standard_normal(len(ri))
    o = rng.permutation(len(ri))
    return ri[o], ci[o], va[o]


@pytest.mark.parametrize("lens", [[6000], [70000, 5, 4097], [12000, 3, 40, 9000]])
def test_long_rows_against_oracle(gpu, O, lens):
    """Rows above one block's sort (4096 keys) take merge passes; 6000 and 70000 need an
    odd number of them, 12000 an even one. Compared with the restatement."""
    rng = np.random.default_rng(sum(lens))
    ri = np.repeat(np.arange(len(lens), dtype=np.int64), lens)
    ci = rng.integers(0, 3000, size=len(ri))  # many duplicates
    va = rng.standard_normal(len(ri))
    o = rng.permutation(len(ri))
    ri, ci, va = ri[o], ci[o], va[o]
    code, want = O.mtx_to_mat("port", len(lens), 3000, ri, ci, va)
    assert code == 0
    _same(gpu.MAT.FromCOO(len(lens), 3000, ri, ci, va), want)


def test_random_large_against_oracle(gpu, O):
    rng = np.random.default_rng(5)
    n = 200_000
    ri, ci, va = _random_coo(rng, n, n, 12)
    code, want = O.mtx_to_mat("port", n, n, ri, ci, va)
    assert code == 0
    _same(gpu.MAT.FromCOO(n, n, ri, ci, va), want)
    # the same entries as raw 1-based CSR with rows in shuffled column order
    o = np.lexsort((rng.random(len(ri)), ri))
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(ri, minlength=n), out=rp[1:])
    code, want = O.csr_to_mat("port", n, rp + 1, ci[o] + 1, va[o])
    assert code == 0
    _same(gpu.MAT.FromCSRRaw(n, rp + 1, ci[o] + 1, va[o]), want)


def test_shuffled_stencil_at_size(gpu):
    """A 64^3 7-point matrix (1.8M entries) from shuffled triplets is the stencil's CSR."""
    A = P.poisson3d(64)
    rows = np.repeat(np.arange(A.nrow, dtype=np.int64), np.diff(A.rowPtr.astype(np.int64)))
    o = np.random.default_rng(9).permutation(A.nnz)
    M = gpu.MAT.FromCOO(A.nrow, A.mcol, rows[o], A.colInd[o], A.values[o])
    _same(M, (A.rowPtr, A.colInd, A.values))
    x = gpu.DVec.from_numpy(np.random.default_rng(1).standard_normal(A.nrow))
    y = gpu.DVec(A.nrow)
    M.Apply(x, y)
    assert np.allclose(y.numpy(), A.matvec(x.numpy()), rtol=1e-14, atol=1e-12)
    assert M.RowClassInfo()[0] == 2  # the stencil form is found as for MAT(csr)


@pytest.mark.parametrize("case", ["row_out_of_range", "col_out_of_range", "rowptr_base",
                                  "rowptr_not_monotone", "nnz_mismatch", "zero_in_1based",
                                  "tall_missing_diag"])
def test_invalid_inputs_rejected(gpu, case):
    from faspxx_b200 import capi
    with pytest.raises(capi.FaspError) as e:
        if case == "row_out_of_range":
            gpu.MAT.FromCOO(3, 3, [0, 3], [0, 1], [1.0, 2.0])
        elif case == "col_out_of_range":
            gpu.MAT.FromCOO(3, 3, [0, 1], [0, 3], [1.0, 2.0])
        elif case == "rowptr_base":
            gpu.MAT.FromCSRRaw(2, [2, 3, 4], [0, 1], [1.0, 2.0])
        elif case == "rowptr_not_monotone":
            gpu.MAT.FromCSRRaw(3, [0, 2, 1, 3], [0, 1, 2], [1.0, 2.0, 3.0])
        elif case == "nnz_mismatch":
            gpu.MAT.FromCSRRaw(2, [0, 1, 3], [0, 1], [1.0, 2.0])
        elif case == "zero_in_1based":
            gpu.MAT.FromCSRRaw(2, [1, 2, 3], [1, 0], [1.0, 2.0])
        else:
            gpu.MAT.FromCOO(3, 2, [0, 1, 2], [0, 1, 0], [1.0, 2.0, 3.0])
    assert e.value.code == -17
    with pytest.raises(capi.FaspError) as e:
        gpu.MAT.FromCOO(3, 3, [], [], [])
    assert e.value.code == -15


def test_solve_on_ingested_matrix(gpu):
    """A matrix built from the raw 1-based, unsorted .csr fixture is a working solver
    operator: weighted-Jacobi PCG drives A x to zero from x0 = 1 (the TestPCG setup)."""
    c = CASES["fdm_10X10_csr"]
    M = gpu.MAT.FromCSRRaw(c["nrow"], *c["inputs"])
    s = gpu.configure("cg", maxIter=100, relTol=1e-6, absTol=0.0, pcd="jacobi", pcdWeight=0.8,
                      pcdIter=1)
    s.Setup(M)
    x = np.ones(c["nrow"])
    assert s.Solve(np.zeros(c["nrow"]), x) == 0
    A = P.CSRMatrix(c["nrow"], c["nrow"], *c["expected"])
    assert np.linalg.norm(A.matvec(x)) < 1e-6 * np.linalg.norm(A.matvec(np.ones(c["nrow"])))
