"""MAT::Mult on the GPU (fasp_gpu_mat_mult).

Bar: bit-exact. Row pointers, column indices (in the reference's first-appearance order,
rows not sorted) and values equal the reference's MAT::Mult on the fixtures
(tests/golden/reference_mult.*) and the oracle's restatement (pinned on the same fixtures)
on larger products: stencil squares, Galerkin triple products with trilinear interpolation,
rectangular random factors with duplicate columns, and rows of more than 4,096
intermediate products (the merge-pass sort).
"""
import numpy as np
import pytest

from faspxx_b200 import problems as P
from tests.golden import cases as G

pytestmark = pytest.mark.gpu

CASES = G.mult_cases()


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    return oracle


def _same(M, want):
    D = M.download()
    for got, w in zip((D.rowPtr, D.colInd, D.values), want):
        assert got.dtype == w.dtype and np.array_equal(got, w)


@pytest.mark.parametrize("name", sorted(CASES))
def test_matches_reference(gpu, name):
    L, R, want = CASES[name]
    C = gpu.MAT(L).Mult(gpu.MAT(R))
    assert (C.GetRowSize(), C.GetColSize()) == (L.nrow, R.mcol)
    _same(C, want)


def _interp1d(nf):
    nc = (nf - 1) // 2
    rows = []
    for i in range(nf):
        if i % 2 == 1:
            rows.append([((i - 1) // 2, 1.0)])
        else:
            r = []
            if i // 2 - 1 >= 0:
                r.append((i // 2 - 1, 0.5))
            if i // 2 < nc:
                r.append((i // 2, 0.5))
            rows.append(r)
    return rows, nc


def _trilinear(nf):
    """Prolongation from a (nf-1)/2 cubed grid to nf cubed, x fastest (Kronecker product)."""
    r1, nc = _interp1d(nf)
    rp, ci, va = [0], [], []
    for k in range(nf):
        for j in range(nf):
            for i in range(nf):
                for (c3, w3) in r1[k]:
                    for (c2, w2) in r1[j]:
                        for (c1, w1) in r1[i]:
                            ci.append(c1 + nc * (c2 + nc * c3))
                            va.append(w1 * w2 * w3)
                rp.append(len(ci))
    return P.CSRMatrix(nf ** 3, nc ** 3, np.array(rp, np.uint32), np.array(ci, np.uint32),
                       np.array(va, np.float64))


def _random(rng, n, m, lo, hi):
    k = rng.integers(lo, hi + 1, size=n)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(k, out=rp[1:])
    ci = rng.integers(0, m, size=int(rp[-1]))
    va = rng.standard_normal(len(ci))
    return P.CSRMatrix(n, m, rp.astype(np.uint32), ci.astype(np.uint32), va)


def test_galerkin_triple_product_against_oracle(gpu, O):
    A = P.poisson3d(15)
    Pm = _trilinear(15)
    Rm = P.CSRMatrix(Pm.mcol, Pm.nrow, *O.transpose("ref", Pm)[:3])
    gA, gP, gR = gpu.MAT(A), gpu.MAT(Pm), gpu.MAT(Rm)
    AP = gA.Mult(gP)
    _same(AP, O.mat_mult("port", A, Pm))
    APc = AP.download()
    Ac = gR.Mult(AP)
    _same(Ac, O.mat_mult("port", Rm, APc))
    # the coarse operator is the Galerkin product: dense check
    dense = Rm.scipy().toarray() @ A.scipy().toarray() @ Pm.scipy().toarray()
    D = Ac.download()
    assert np.allclose(D.scipy().toarray(), dense, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("shape", [(300, 200, 250, 1, 9), (40, 600, 50, 150, 220)])
def test_random_products_against_oracle(gpu, O, shape):
    """Random factors with repeated columns; the second has rows of up to 220 x 60 = 13,200
    intermediate products (segment sorts and merge passes)."""
    n, k, m, lo, hi = shape
    rng = np.random.default_rng(n + k)
    L = _random(rng, n, k, lo, hi)
    R = _random(rng, k, m, 0, 60 if lo > 1 else 12)
    _same(gpu.MAT(L).Mult(gpu.MAT(R)), O.mat_mult("port", L, R))


def test_stencil_square_at_size(gpu, O):
    A = P.poisson3d(32)
    _same(gpu.MAT(A).Mult(gpu.MAT(A)), O.mat_mult("port", A, A))


def test_errors(gpu):
    from faspxx_b200 import capi
    A, B = gpu.MAT(P.poisson2d(5)), gpu.MAT(P.poisson2d(6))
    with pytest.raises(capi.FaspError) as e:
        A.Mult(B)
    assert e.value.code == -16
    S = gpu.MAT.Stencil((5, 5), [((0, 0), 2.0), ((1, 0), -1.0)])
    with pytest.raises(capi.FaspError) as e:
        S.Mult(A)
    assert e.value.code == -12
    pat = P.poisson2d(5)
    with pytest.raises(capi.FaspError) as e:
        gpu.MAT(P.CSRMatrix(pat.nrow, pat.mcol, pat.rowPtr, pat.colInd, None)).Mult(A)
    assert e.value.code == -12


ADD = G.add_cases()


@pytest.mark.parametrize("name", sorted(ADD))
def test_add_matches_reference(gpu, name):
    a, A, b, B, want = ADD[name]
    _same(gpu.MAT.Add(a, gpu.MAT(A), b, gpu.MAT(B)), want)


def test_add_at_size_against_oracle(gpu, O):
    A = P.poisson3d(24)
    rng = np.random.default_rng(11)
    B = _random(rng, A.nrow, A.mcol, 1, 5)
    # row 0 of B starts with column 0 (the reference's sort cannot front-load row 0)
    B.colInd[B.rowPtr[0]] = 0
    code, want = O.mat_add("port", 0.75, A, -2.5, B)
    assert code == 0
    _same(gpu.MAT.Add(0.75, gpu.MAT(A), -2.5, gpu.MAT(B)), want)


def test_add_errors(gpu):
    from faspxx_b200 import capi
    with pytest.raises(capi.FaspError) as e:
        gpu.MAT.Add(1.0, gpu.MAT(P.poisson2d(5)), 1.0, gpu.MAT(P.poisson2d(6)))
    assert e.value.code == -16
