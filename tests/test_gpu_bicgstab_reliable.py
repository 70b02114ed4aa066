"""BiCGStab with reliable updates (MIXED_RELIABLE): FP32 iterations, FP64 answers.

No reference counterpart (FASP++ computes in FP64 only); held to the FP64 BiCGStab's
contract on the same inputs:

* code 0 means the FP64 true residual ||b - A x|| / ||b - A x0|| is below relTol (checked
  here in numpy from the returned x);
* the solution agrees with the FP64 BiCGStab solution within 1e-5 of max|x| at relTol 1e-8;
* the Krylov process survives each refresh (p and r0* are kept), so the iteration count
  stays near FP64 BiCGStab's, unlike restarted refinement (MIXED);
* History()[0] is ||b - A x0||, the entry at the last iteration the final FP64 residual;
* maxIter reached without convergence returns ERROR_SOLVER_MAXIT (-39); a solve that
  starts converged makes no iteration.
"""
import numpy as np
import pytest

from faspxx_b200 import problems as P

pytestmark = pytest.mark.gpu

MAXIT = -39


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


def _solver(gpu, A, prec, jac=True, relTol=1e-8, maxIter=3000, delta=None, M=None):
    from faspxx_b200 import capi
    s = gpu.configure("bicgstab", maxIter=maxIter, relTol=relTol, absTol=0.0,
                      pcd="jacobi" if jac else None, pcdWeight=2.0 / 3.0, pcdIter=1)
    if prec != "FP64":
        s.SetPrecision(getattr(capi, prec), innerRelTol=delta)
    s.Setup(M if M is not None else gpu.MAT(A))
    return s


@pytest.mark.parametrize("pe", [0.1, 10.0])
@pytest.mark.parametrize("jac", [True, False])
def test_reliable_meets_fp64_contract(gpu, pe, jac):
    A = P.convdiff3d(24, pe)
    rng = np.random.default_rng(7)
    xs = rng.uniform(-1.0, 1.0, A.nrow)
    b = A.matvec(xs)
    x0 = rng.standard_normal(A.nrow) * 0.1
    ref = _solver(gpu, A, "FP64", jac)
    xr = x0.copy()
    assert ref.Solve(b, xr) == 0
    s = _solver(gpu, A, "MIXED_RELIABLE", jac)
    x = x0.copy()
    code = s.Solve(b, x)
    assert code == 0, code
    r0 = np.linalg.norm(b - A.matvec(x0))
    rel = np.linalg.norm(b - A.matvec(x)) / r0
    assert rel < 1e-8, rel
    assert np.max(np.abs(x - xr)) <= 1e-5 * np.max(np.abs(xr))
    h = s.History()
    it, it64 = s.GetIterations(), ref.GetIterations()
    assert abs(h[0] - r0) <= 1e-12 * r0
    assert abs(h[it] - rel * r0) <= 1e-6 * rel * r0
    assert it <= it64 * 1.25 + 5, (it, it64)
    assert s.info.outerIter >= 2  # at least one delta refresh and the final check


@pytest.mark.parametrize("delta", [0.5, 1e-1, 1e-3])
def test_reliable_delta_sweep(gpu, delta):
    A = P.convdiff3d(20, 1.0)
    b = A.matvec(np.random.default_rng(3).uniform(-1, 1, A.nrow))
    s = _solver(gpu, A, "MIXED_RELIABLE", delta=delta)
    x = np.zeros(A.nrow)
    assert s.Solve(b, x) == 0
    assert np.linalg.norm(b - A.matvec(x)) < 1e-8 * np.linalg.norm(b)


def test_reliable_csr_form_and_stencil_form_agree(gpu):
    """The FP32 engine runs the stencil-mask kernels on a constant-coefficient matrix and
    the CSR ones otherwise: both forms reach the tolerance with the same iteration count
    (each row's product is the same bits in either form)."""
    A = P.convdiff3d(16, 10.0)
    b = A.matvec(np.random.default_rng(5).uniform(-1, 1, A.nrow))
    out = []
    for form in (0, 2):
        M = gpu.MAT(A)
        M.SetRowClass(form)
        s = _solver(gpu, A, "MIXED_RELIABLE", M=M)
        x = np.zeros(A.nrow)
        assert s.Solve(b, x) == 0
        out.append((s.GetIterations(), x))
    assert np.linalg.norm(b - A.matvec(out[0][1])) < 1e-8 * np.linalg.norm(b)
    assert abs(out[0][0] - out[1][0]) <= 2


def test_reliable_maxit(gpu):
    A = P.convdiff3d(20, 1.0)
    b = A.matvec(np.random.default_rng(9).uniform(-1, 1, A.nrow))
    s = _solver(gpu, A, "MIXED_RELIABLE", maxIter=5)
    x = np.zeros(A.nrow)
    assert s.Solve(b, x) == MAXIT
    assert s.GetIterations() == 5
    # the returned x is the FP64 fold of the five FP32 steps: better than x0 = 0
    assert np.linalg.norm(b - A.matvec(x)) < np.linalg.norm(b)


def test_reliable_starts_converged(gpu):
    A = P.convdiff3d(12, 1.0)
    xs = np.random.default_rng(2).uniform(-1, 1, A.nrow)
    b = A.matvec(xs)
    from faspxx_b200 import capi
    s = gpu.configure("bicgstab", maxIter=100, relTol=1e-8, absTol=1e-10, pcd="jacobi",
                      pcdWeight=2.0 / 3.0, pcdIter=1)
    s.SetPrecision(capi.MIXED_RELIABLE)
    s.Setup(gpu.MAT(A))
    x = xs.copy()
    assert s.Solve(b, x) == 0  # ||b - A x*|| is rounding, below absTol
    assert s.GetIterations() == 0
    assert np.array_equal(x, xs)


def test_reliable_rejects_unfused_preconditioner(gpu):
    """Reliable updates run in the fused FP32 engine: a multi-sweep Jacobi is refused."""
    from faspxx_b200 import capi
    A = P.convdiff3d(10, 1.0)
    s = gpu.configure("bicgstab", maxIter=100, relTol=1e-8, absTol=0.0, pcd="jacobi",
                      pcdIter=3)
    s.SetPrecision(capi.MIXED_RELIABLE)
    with pytest.raises(Exception):
        s.Setup(gpu.MAT(A))


def _row_scaled(A, seed):
    """S A with S = diag(10^U(-1, 1)): nonsymmetric, and its diagonal varies row to row."""
    rng = np.random.default_rng(seed)
    scale = 10.0 ** rng.uniform(-1.0, 1.0, A.nrow)
    rows = np.repeat(np.arange(A.nrow), np.diff(A.rowPtr.astype(np.int64)))
    return P.CSRMatrix(A.nrow, A.mcol, A.rowPtr, A.colInd, A.values * scale[rows])


@pytest.mark.parametrize("pe", [0.1, 10.0])
def test_reliable_variable_diagonal(gpu, pe):
    """With a diagonal that varies, the FP32 engine applies Jacobi on the right (A (D p)), so
    that its recursive residual is b - A x and each refresh replaces it consistently: the
    solve meets the FP64 tolerance and agrees with a sparse direct solve."""
    A = _row_scaled(P.convdiff3d(20, pe), 4)
    rng = np.random.default_rng(8)
    xs = rng.uniform(-1.0, 1.0, A.nrow)
    b = A.matvec(xs)
    s = _solver(gpu, A, "MIXED_RELIABLE")
    x = np.zeros(A.nrow)
    code = s.Solve(b, x)
    assert code == 0, code
    rel = np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)
    assert rel < 1e-8, rel
    assert s.info.outerIter >= 2
    import scipy.sparse.linalg as sla
    xd = sla.spsolve(A.scipy().tocsc(), b)
    assert np.max(np.abs(x - xd)) <= 1e-5 * np.max(np.abs(xd))
