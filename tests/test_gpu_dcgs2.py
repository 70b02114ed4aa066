"""GMRES with the reorthogonalisation delayed into the next Arnoldi step (ORTH_DCGS2).

DCGS2 computes the same Arnoldi process as CGS2 (classical Gram-Schmidt with one
reorthogonalisation) with two passes over the basis per step instead of three. Held here to
CGS2's results on the same inputs, and to the true residual:

* same return code; iteration count within one of CGS2's; solutions agree to 1e-6 of
  max|x| at relTol 1e-8; the true residual meets the tolerance (x checked in numpy);
* the streamed passes cut vectors into 12 KB chunks over contiguous block ranges: sizes
  from 1 to a few chunks per block, odd (FP64) and non-multiple-of-4 (FP32) lengths;
* reruns give identical bits; a restart length above 48 runs as CGS2 (bit-identical to it);
* maxIter inside a restart cycle, variable restart, left preconditioning, no
  preconditioner and the FP32 inner solves of MIXED.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from faspxx_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return capi, sol


def _run(gpu, A, b, orth, alg="gmres", pcd="jacobi", prec="FP64", x0=None, **kw):
    capi, sol = gpu
    args = dict(maxIter=2000, relTol=1e-8, absTol=0.0, restart=30, pcd=pcd,
                pcdWeight=2.0 / 3.0, pcdIter=1)
    args.update(kw)
    s = sol.configure(alg, **args)
    s.SetOrth(getattr(capi, "ORTH_" + orth.upper()))
    if prec != "FP64":
        s.SetPrecision(getattr(capi, prec))
    s.Setup(sol.MAT(A))
    x = np.zeros(A.nrow) if x0 is None else x0.copy()
    code = s.Solve(b, x)
    return code, s.GetIterations(), x, s.History()


def _convection_1d(n, seed):
    """Tridiagonal upwind convection-diffusion with a varying diagonal: nonsymmetric, any n."""
    rng = np.random.default_rng(seed)
    d = 2.5 + rng.uniform(0.0, 1.0, n)
    A = sp.diags([np.full(n - 1, -1.3), d, np.full(n - 1, -0.7)], [-1, 0, 1], format="csr")
    A.sort_indices()
    return P.CSRMatrix(n, n, A.indptr.astype(np.int32), A.indices.astype(np.int32),
                       A.data.astype(np.float64))


def _agree(A, b, r_dcgs2, r_cgs2, tol=1e-8, xtol=1e-6):
    code, it, x, _ = r_dcgs2
    code2, it2, x2, _ = r_cgs2
    assert code == code2, (code, code2)
    assert abs(it - it2) <= 1, (it, it2)
    r0 = np.linalg.norm(b)
    assert np.linalg.norm(b - A.matvec(x)) <= 10 * tol * r0
    assert np.max(np.abs(x - x2)) <= xtol * max(np.max(np.abs(x2)), 1e-300)


@pytest.mark.parametrize("alg", ["gmres", "gmres_left"])
@pytest.mark.parametrize("pcd", [None, "jacobi"])
@pytest.mark.parametrize("pe", [0.1, 10.0])
def test_dcgs2_matches_cgs2(gpu, alg, pcd, pe):
    A = P.convdiff3d(16, pe)
    b = A.matvec(np.random.default_rng(1).uniform(-1, 1, A.nrow))
    _agree(A, b, _run(gpu, A, b, "dcgs2", alg=alg, pcd=pcd),
           _run(gpu, A, b, "cgs2", alg=alg, pcd=pcd))


@pytest.mark.parametrize("prec", ["FP64", "MIXED"])
@pytest.mark.parametrize("n", [1, 2, 3, 7, 61, 1001, 4099, 20001, 1000003])
def test_dcgs2_ragged_sizes(gpu, n, prec):
    """Lengths below one group, below one chunk, and several chunks per block, all odd:
    the last group of the last block is partial in FP64 and FP32 alike."""
    A = _convection_1d(n, n)
    b = np.random.default_rng(n).standard_normal(n)
    r = _run(gpu, A, b, "dcgs2", prec=prec)
    assert r[0] == 0, r[0]
    assert np.linalg.norm(b - A.matvec(r[2])) <= 1e-7 * np.linalg.norm(b)
    _agree(A, b, r, _run(gpu, A, b, "cgs2", prec=prec), tol=1e-8 if prec == "FP64" else 1e-7,
           xtol=1e-6)


def test_dcgs2_deterministic(gpu):
    A = P.convdiff3d(20, 1.0)
    b = A.matvec(np.random.default_rng(4).uniform(-1, 1, A.nrow))
    r1 = _run(gpu, A, b, "dcgs2")
    r2 = _run(gpu, A, b, "dcgs2")
    assert r1[1] == r2[1]
    assert np.array_equal(r1[2], r2[2])
    assert np.array_equal(r1[3], r2[3], equal_nan=True)


def test_dcgs2_long_restart_runs_cgs2(gpu):
    """A restart length above the 48 vectors the delayed passes take runs as CGS2."""
    A = P.convdiff3d(16, 10.0)
    b = A.matvec(np.random.default_rng(5).uniform(-1, 1, A.nrow))
    r1 = _run(gpu, A, b, "dcgs2", restart=60, maxRestart=60, minRestart=60)
    r2 = _run(gpu, A, b, "cgs2", restart=60, maxRestart=60, minRestart=60)
    assert r1[0] == r2[0] and r1[1] == r2[1]
    assert np.array_equal(r1[2], r2[2])


@pytest.mark.parametrize("maxIter", [1, 17, 45])
def test_dcgs2_maxiter_inside_a_cycle(gpu, maxIter):
    A = P.convdiff3d(16, 10.0)
    b = A.matvec(np.random.default_rng(6).uniform(-1, 1, A.nrow))
    c1, i1, x1, h1 = _run(gpu, A, b, "dcgs2", maxIter=maxIter)
    c2, i2, x2, h2 = _run(gpu, A, b, "cgs2", maxIter=maxIter)
    assert (c1, i1) == (c2, i2)
    assert np.max(np.abs(x1 - x2)) <= 1e-9 * np.max(np.abs(x2))
    m = min(len(h1), len(h2))
    fin = np.isfinite(h2[:m])
    assert np.array_equal(fin, np.isfinite(h1[:m]))
    assert np.all(np.abs(h1[:m][fin] - h2[:m][fin]) <= 1e-9 * h2[:m][fin])


def test_dcgs2_variable_restart(gpu):
    """The reference's default restart range (30 down to 10 by 3, GMRES.cxx:255-265)."""
    A = P.convdiff3d(20, 10.0)
    b = A.matvec(np.random.default_rng(7).uniform(-1, 1, A.nrow))
    _agree(A, b, _run(gpu, A, b, "dcgs2", maxRestart=30, minRestart=10),
           _run(gpu, A, b, "cgs2", maxRestart=30, minRestart=10))


@pytest.mark.parametrize("pe", [0.1, 10.0])
def test_dcgs2_mixed_precision(gpu, pe):
    """FP32 inner GMRES cycles inside FP64 refinement: the FP64 answer and tolerance."""
    A = P.convdiff3d(24, pe)
    xs = np.random.default_rng(8).uniform(-1, 1, A.nrow)
    b = A.matvec(xs)
    c1, i1, x1, _ = _run(gpu, A, b, "dcgs2", prec="MIXED")
    c2, i2, x2, _ = _run(gpu, A, b, "cgs2", prec="MIXED")
    assert c1 == 0 and c2 == 0
    assert np.linalg.norm(b - A.matvec(x1)) <= 1e-8 * np.linalg.norm(b)
    assert abs(i1 - i2) <= max(3, 0.05 * i2), (i1, i2)
    # relTol 1e-8 bounds the residual, not the error: the error against x* is CGS2's
    e1, e2 = np.max(np.abs(x1 - xs)), np.max(np.abs(x2 - xs))
    assert e1 <= 2.0 * e2 + 1e-9 * np.max(np.abs(xs)), (e1, e2)


def _upwind_2d(nx, pe):
    """A nonsymmetric 5-point operator on an nx x nx grid: the 2D Laplacian plus first-order
    upwind convection along x (the 5-point shape of the stencil-mask product)."""
    A = P.poisson2d(nx)
    rows = np.repeat(np.arange(A.nrow), np.diff(A.rowPtr.astype(np.int64)))
    vals = A.values.copy()
    d = A.colInd.astype(np.int64) - rows
    vals[d == 0] += pe
    vals[d == -1] -= pe
    return P.CSRMatrix(A.nrow, A.mcol, A.rowPtr, A.colInd, vals)


@pytest.mark.parametrize("alg", ["gmres", "gmres_left"])
@pytest.mark.parametrize("shape", ["7-point", "5-point"])
def test_dcgs2_fused_product_same_bits(gpu, alg, shape):
    """The FP32 cycles form the product inside the dots pass on stencil masks of the fixed
    5- or 7-point shape; on plain CSR the product is a separate kernel. Both give each row's
    sum with the same operations: the mixed solves agree bit for bit, at a size with several
    blocks and block ranges that end inside a warp's groups."""
    capi, sol = gpu
    A = P.convdiff3d(40, 10.0) if shape == "7-point" else _upwind_2d(300, 0.5)
    b = A.matvec(np.random.default_rng(9).uniform(-1, 1, A.nrow))
    out = []
    for form in (0, 2):  # plain CSR, stencil masks
        M = sol.MAT(A)
        M.SetRowClass(form)
        s = sol.configure(alg, maxIter=3000, relTol=1e-8, absTol=0.0, restart=30, pcd="jacobi",
                          pcdWeight=2.0 / 3.0, pcdIter=1)
        s.SetPrecision(capi.MIXED)
        s.Setup(M)
        x = np.zeros(A.nrow)
        code = s.Solve(b, x)
        out.append((code, s.GetIterations(), x))
    assert out[0][0] == out[1][0] == 0
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
    assert np.linalg.norm(b - A.matvec(out[1][2])) <= 1e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("prec", ["FP64", "MIXED"])
def test_dcgs2_restart_48(gpu, prec):
    """The longest restart the delayed passes take (48 basis vectors: 98 values in one dots
    reduction), against CGS2 on the same system."""
    A = P.convdiff3d(32, 10.0)
    b = A.matvec(np.random.default_rng(11).uniform(-1, 1, A.nrow))
    kw = dict(restart=48, maxRestart=48, minRestart=48, prec=prec)
    _agree(A, b, _run(gpu, A, b, "dcgs2", **kw), _run(gpu, A, b, "cgs2", **kw),
           tol=1e-8, xtol=1e-6 if prec == "FP64" else 1e-5)
