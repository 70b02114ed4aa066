"""MAT::MultTransposeAdd (src/MAT.cxx:541-606), v = A^T v1 + v2: the oracle's restatement
against the reference's recorded results (tests/golden/reference_mta.*).

On structurally symmetric matrices the restatement reproduces the reference bit for bit
(v starts from v2, each column's products are added in ascending row order, rounded one at
a time). On a matrix whose row pointers differ from its transpose's, the reference bounds
each column by A's own rowPtr (MAT.cxx:603) and its result is not A^T v1 + v2; the
restatement (and the GPU) use the transpose's bounds, checked against a dense product.
"""
import numpy as np
import pytest

from tests.golden import cases as G


@pytest.fixture(scope="module")
def oracle():
    from oracle import oracle as O
    O.build(ref=False)
    return O


@pytest.mark.parametrize("name", sorted(G.mta_cases()))
def test_restatement_matches_reference(oracle, name):
    A, v1, v2, vref, sym = G.mta_cases()[name]
    code, v = oracle.mult_transpose_add("port", A, v1, v2)
    assert code == 0
    dense = A.scipy().T @ v1 + v2
    assert np.allclose(v, dense, rtol=1e-13, atol=1e-13 * np.abs(dense).max())
    if sym:
        assert np.array_equal(v.view(np.uint64), vref.view(np.uint64)), name
    else:
        # the reference's loop bound (MAT.cxx:603) gives another vector here
        assert not np.allclose(vref, dense, rtol=1e-6, atol=1e-6), name


def test_rectangular_and_pattern(oracle):
    """Cases the reference cannot run (its loop reads past A's rowPtr, or reads an empty
    values array): the restatement against dense products; pattern entries count as 1."""
    from faspxx_b200 import problems as P
    rng = np.random.default_rng(8)
    n, m = 30, 45
    dense = (rng.random((n, m)) < 0.15) * rng.standard_normal((n, m))
    for i in range(n):
        dense[i, i] = 1.0 + i
    import scipy.sparse as sp
    S = sp.csr_matrix(dense)
    S.sort_indices()
    A = P.CSRMatrix(n, m, S.indptr.astype(np.uint32), S.indices.astype(np.uint32), S.data)
    v1, v2 = rng.standard_normal(n), rng.standard_normal(m)
    code, v = oracle.mult_transpose_add("port", A, v1, v2)
    assert code == 0 and np.allclose(v, dense.T @ v1 + v2, rtol=1e-13, atol=1e-13)
    Pat = P.CSRMatrix(n, m, A.rowPtr, A.colInd, None)
    code, v = oracle.mult_transpose_add("port", Pat, v1, v2)
    assert code == 0 and np.allclose(v, (dense != 0).T @ v1 + v2, rtol=1e-13, atol=1e-13)
