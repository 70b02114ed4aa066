"""Mixed-precision CG on the GPU: FP32 Krylov iterations, FP64 answers.

Neither mode has a reference counterpart (FASP++ computes in FP64 only); both are held to
the FP64 solver's contract on the same inputs:

* the FP64 true residual ||b - A x|| / ||b - A x0|| is below relTol when code 0 is returned
  (checked here in numpy from the returned x);
* the solution agrees with the FP64 CG solution within cond-scaled relTol (1e-5 relative
  to max|x| at relTol 1e-8 on these problems);
* MIXED_RELIABLE keeps the Krylov process across its FP64 refreshes, so its iteration
  count stays within 5% (+2) of FP64 CG's; restarted refinement (MIXED) may take more;
* History()[0] is ||b - A x0|| and the last entry is the final FP64 true residual;
* maxIter reached without convergence returns ERROR_SOLVER_MAXIT (-39).
"""
import numpy as np
import pytest

from faspxx_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


def _solver(gpu, A, precision, jac=True, relTol=1e-8, maxIter=2000, delta=None):
    from faspxx_b200 import capi
    s = gpu.CG()
    s.SetMaxIter(maxIter)
    s.SetRelTol(relTol)
    s.SetAbsTol(0.0)
    if jac:
        pc = gpu.Jacobi()
        pc.SetMaxIter(1)
        pc.SetMinIter(1)
        s.SetupPCD(pc)
    if precision != capi.FP64:
        s.SetPrecision(precision, innerRelTol=delta)
    s.Setup(gpu.MAT(A))
    return s


def _vardiff(N, seed=11):
    # log-uniform cell coefficients over two decades
    kappa = 10.0 ** np.random.default_rng(seed).uniform(-1.0, 1.0, N ** 3)
    return P.vardiff3d(N, kappa)


def _problems():
    return {
        "poisson3d_32": P.poisson3d(32),
        "vardiff3d_24": _vardiff(24),
    }


@pytest.mark.parametrize("name", ["poisson3d_32", "vardiff3d_24"])
@pytest.mark.parametrize("jac", [True, False])
@pytest.mark.parametrize("mode", ["MIXED", "MIXED_RELIABLE"])
def test_mixed_meets_fp64_contract(gpu, name, jac, mode):
    from faspxx_b200 import capi
    A = _problems()[name]
    rng = np.random.default_rng(7)
    xs = rng.uniform(0.0, 1.0, A.nrow)
    b = A.matvec(xs)
    x0 = rng.standard_normal(A.nrow) * 0.1
    ref = _solver(gpu, A, capi.FP64, jac)
    xr = x0.copy()
    assert ref.Solve(b, xr) == 0
    s = _solver(gpu, A, getattr(capi, mode), jac)
    x = x0.copy()
    code = s.Solve(b, x)
    assert code == 0, code
    r0 = np.linalg.norm(b - A.matvec(x0))
    rel = np.linalg.norm(b - A.matvec(x)) / r0
    assert rel < 1e-8, rel
    assert np.max(np.abs(x - xr)) <= 1e-5 * np.max(np.abs(xr))
    h = s.History()
    assert abs(h[0] - r0) <= 1e-12 * r0
    assert abs(h[s.GetIterations()] - rel * r0) <= 1e-6 * rel * r0
    if mode == "MIXED_RELIABLE":
        it, it64 = s.GetIterations(), ref.GetIterations()
        assert it <= it64 * 1.05 + 2, (it, it64)
        assert s.info.outerIter >= 2  # at least one delta refresh and the final check


@pytest.mark.parametrize("delta", [0.5, 1e-1, 1e-3])
def test_reliable_delta_sweep(gpu, delta):
    """Every refresh factor converges to the FP64 tolerance."""
    from faspxx_b200 import capi
    A = P.poisson3d(24)
    b = A.matvec(np.random.default_rng(3).uniform(0, 1, A.nrow))
    s = _solver(gpu, A, capi.MIXED_RELIABLE, delta=delta)
    x = np.zeros(A.nrow)
    assert s.Solve(b, x) == 0
    assert np.linalg.norm(b - A.matvec(x)) < 1e-8 * np.linalg.norm(b)


def test_reliable_maxit_and_converged_start(gpu):
    from faspxx_b200 import capi
    A = P.poisson3d(24)
    xs = np.random.default_rng(5).uniform(0, 1, A.nrow)
    b = A.matvec(xs)
    s = _solver(gpu, A, capi.MIXED_RELIABLE, maxIter=10)
    x = np.zeros(A.nrow)
    assert s.Solve(b, x) == -39
    assert s.GetIterations() == 10
    # the FP64 residual of the returned x is the one reported
    assert abs(s.info.norm2 - np.linalg.norm(b - A.matvec(x))) <= 1e-9 * s.info.norm2
    # a start that already meets the absolute tolerance: no iterations
    s2 = _solver(gpu, A, capi.MIXED_RELIABLE)
    s2.SetAbsTol(1e-6)
    s2.Setup(s2.A)
    x = xs.copy()
    assert s2.Solve(b, x) == 0
    assert s2.GetIterations() == 0
    assert np.array_equal(x, xs)


def test_reliable_repeat_solves_are_deterministic(gpu):
    from faspxx_b200 import capi
    A = _vardiff(20)
    b = A.matvec(np.ones(A.nrow))
    s = _solver(gpu, A, capi.MIXED_RELIABLE)
    xa, xb = np.zeros(A.nrow), np.zeros(A.nrow)
    s.Solve(b, xa)
    ia = s.GetIterations()
    s.Solve(b, xb)
    assert s.GetIterations() == ia
    assert np.array_equal(xa, xb)


# ---- mixed-precision BiCGStab / GMRES / FGMRES: FP64 refinement around FP32 inner solves ----

KRYLOV = ["bicgstab", "gmres", "gmres_left", "fgmres"]


def _krylov(gpu, alg, A, precision, relTol=1e-8):
    from faspxx_b200 import capi
    kw = dict(maxIter=3000, relTol=relTol, absTol=0.0, pcd="jacobi", pcdWeight=2.0 / 3.0,
              pcdIter=1)
    if alg != "bicgstab":
        kw.update(restart=30, maxRestart=30, minRestart=10)
    s = gpu.configure(alg, **kw)
    if precision != capi.FP64:
        s.SetPrecision(precision, innerRelTol=1e-4)
    s.Setup(gpu.MAT(A))
    return s


@pytest.mark.parametrize("peclet", [0.1, 10.0])
@pytest.mark.parametrize("alg", KRYLOV)
def test_mixed_krylov_refinement(gpu, alg, peclet):
    """FP32 inner iterations (FP64 Hessenberg/Givens for the GMRES family) inside FP64
    refinement reach the FP64 tolerance on the upwind convection-diffusion matrices."""
    from faspxx_b200 import capi
    A = P.convdiff3d(20, peclet)
    rng = np.random.default_rng(13)
    xs = rng.uniform(-1.0, 1.0, A.nrow)
    b = A.matvec(xs)
    ref = _krylov(gpu, alg, A, capi.FP64)
    xr = np.zeros(A.nrow)
    assert ref.Solve(b, xr) == 0
    s = _krylov(gpu, alg, A, capi.MIXED)
    x = np.zeros(A.nrow)
    assert s.Solve(b, x) == 0
    rel = np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)
    assert rel < 1e-8, rel
    assert np.max(np.abs(x - xr)) <= 1e-5 * np.max(np.abs(xr))
    assert s.info.outerIter >= 2
    h = s.History()
    assert abs(h[0] - np.linalg.norm(b)) <= 1e-12 * np.linalg.norm(b)
    assert abs(h[s.GetIterations()] - rel * np.linalg.norm(b)) <= 1e-6 * rel * np.linalg.norm(b)


def test_mixed_precision_rejected_for_stationary_solvers(gpu):
    from faspxx_b200 import capi
    A = P.poisson3d(8)
    for alg in ("jacobi", "mg"):
        s = gpu.configure(alg, maxIter=10)
        s.SetPrecision(capi.MIXED)
        with pytest.raises(capi.FaspError) as e:
            s.Setup(gpu.MAT(A))
        assert e.value.code == -30
    for alg in ("gmres", "fgmres"):  # reliable updates: CG and BiCGStab only
        s = gpu.configure(alg, maxIter=10)
        s.SetPrecision(capi.MIXED_RELIABLE)
        with pytest.raises(capi.FaspError) as e:
            s.Setup(gpu.MAT(A))
        assert e.value.code == -30


def test_reliable_stops_below_attainable_accuracy(gpu):
    """A start already at the rounding floor (x0 = x*): the relative target 1e-10 of a
    residual that is itself rounding noise cannot be met; the FP64 refreshes stop gaining
    and the solve ends with ERROR_SOLVER_TOLSMALL long before maxIter."""
    from faspxx_b200 import capi
    A = P.poisson3d(24)
    xs = np.random.default_rng(9).uniform(0, 1, A.nrow)
    b = A.matvec(xs)
    s = _solver(gpu, A, capi.MIXED_RELIABLE, relTol=1e-10, maxIter=5000)
    x = xs.copy()
    code = s.Solve(b, x)
    assert code in (0, -34), code
    assert s.GetIterations() < 1000
    assert np.max(np.abs(x - xs)) < 1e-10


@pytest.mark.parametrize("rec", [True, False])
@pytest.mark.parametrize("name", ["poisson3d_32", "vardiff3d_24"])
def test_reliable_q_recurrence_and_reference_form(gpu, name, rec):
    """The FP32 iterations reach the FP64 tolerance in the FP64 iteration count (+5%) both
    with the q = A z + beta q_old recurrence (default) and with the reference's A (z + beta
    p) form."""
    from faspxx_b200 import capi
    A = _problems()[name]
    b = A.matvec(np.random.default_rng(21).uniform(0.0, 1.0, A.nrow))
    ref = _solver(gpu, A, capi.FP64)
    xr = np.zeros(A.nrow)
    assert ref.Solve(b, xr) == 0
    s = gpu.CG()
    s.SetMaxIter(2000)
    s.SetRelTol(1e-8)
    s.SetAbsTol(0.0)
    pc = gpu.Jacobi()
    pc.SetMaxIter(1)
    pc.SetMinIter(1)
    s.SetupPCD(pc)
    s.SetPrecision(capi.MIXED_RELIABLE)
    s.SetFP32Recurrence(rec)
    s.Setup(gpu.MAT(A))
    x = np.zeros(A.nrow)
    assert s.Solve(b, x) == 0
    assert np.linalg.norm(b - A.matvec(x)) < 1e-8 * np.linalg.norm(b)
    assert s.GetIterations() <= ref.GetIterations() * 1.05 + 2
