"""MAT::MultTransposeAdd on the GPU (fasp_gpu_mat_mult_transpose_add), v = A^T v1 + v2.

Bars: bit for bit the reference's result (tests/golden/reference_mta.*) on structurally
symmetric matrices, where the reference's loop bounds are right (MAT.cxx:603); bit for
bit the oracle's restatement (the transpose's own bounds) on the structurally
nonsymmetric, rectangular and pattern-only matrices the reference gets wrong or cannot
run; a grid operator bit for bit its assembled matrix. The GPU rounds each product before
adding it, as the reference does, so no tolerance is needed.
"""
import numpy as np
import pytest

from tests.golden import cases as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


def _gpu_mta(sol, M, v1, v2):
    out = sol.DVec(len(v2))
    M.MultTransposeAdd(sol.DVec.from_numpy(v1), sol.DVec.from_numpy(v2), out)
    return out.numpy()


def _bits(a):
    return np.ascontiguousarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("name", sorted(G.mta_cases()))
def test_matches_reference(gpu, name):
    from oracle import oracle as O
    A, v1, v2, vref, sym = G.mta_cases()[name]
    M = gpu.MAT(A)
    for _ in range(2):  # the second call reuses the cached transpose
        v = _gpu_mta(gpu, M, v1, v2)
        if sym:
            assert np.array_equal(_bits(v), _bits(vref)), name
        else:
            _, vport = O.mult_transpose_add("port", A, v1, v2)
            assert np.array_equal(_bits(v), _bits(vport)), name


def test_rectangular_pattern_and_grid(gpu):
    import scipy.sparse as sp
    from faspxx_b200 import problems as P
    from oracle import oracle as O
    rng = np.random.default_rng(8)
    n, m = 300, 451
    dense = (rng.random((n, m)) < 0.02) * rng.standard_normal((n, m))
    S = sp.csr_matrix(dense)
    S.sort_indices()
    A = P.CSRMatrix(n, m, S.indptr.astype(np.uint32), S.indices.astype(np.uint32), S.data)
    v1, v2 = rng.standard_normal(n), rng.standard_normal(m)
    for mat in (A, P.CSRMatrix(n, m, A.rowPtr, A.colInd, None)):
        _, vport = O.mult_transpose_add("port", mat, v1, v2)
        assert np.array_equal(_bits(_gpu_mta(gpu, gpu.MAT(mat), v1, v2)), _bits(vport))
    # a nonsymmetric grid operator (upwind-like 3D stencil) against its assembled matrix
    pts = [((0, 0, -1), -0.6), ((0, -1, 0), -1.1), ((-1, 0, 0), -1.4), ((0, 0, 0), 6.3),
           ((1, 0, 0), -0.9), ((0, 1, 0), -1.2), ((0, 0, 1), -0.8)]
    G3 = gpu.MAT.Stencil((13, 11, 9), pts)
    C = G3.download()
    w1, w2 = rng.standard_normal(C.nrow), rng.standard_normal(C.mcol)
    _, vport = O.mult_transpose_add("port", C, w1, w2)
    assert np.array_equal(_bits(_gpu_mta(gpu, G3, w1, w2)), _bits(vport))
