"""Bad inputs and failure detection on the GPU, all made on the host side (no GPU fault,
trap or endless wait is provoked).

1. The device-driven and host-orchestrated solvers meet NaN/Inf in b, NaN in x0, a zero
   diagonal under Jacobi, maxIter = 1, b = x0 = 0 and a zero matrix (every dot zero) with
   the reference's outcome (tests/golden/cases.py: fault_cases, pinned against the
   reference by tests/test_faults_cpu.py): the same FaspRetCode (CG.cxx:105-119,
   BiCGStab.cxx:118-124), the same iteration count, a NaN residual norm exactly where the
   reference's is NaN, and the same finite/non-finite pattern of x (values within 1e-12 of
   max|x| where finite). CG runs every engine (CUDA graphs, graphs without overlapped
   launches, plain launches, the persistent cooperative kernel).
2. The mixed-precision modes stop on the same inputs in bounded time with a failure code
   or a NaN norm (they have no reference counterpart).
3. The persistent CG's software grid barrier gives up after a configured number of polls:
   with a limit of one poll the solve returns FASP_GPU_ERROR_CUDA (the blocks leave on the
   error flag), and the same solver object then solves normally with the default limit.
"""
import numpy as np
import pytest

from tests.golden import cases as G

pytestmark = pytest.mark.gpu

CASES = G.fault_cases()


@pytest.fixture(scope="module")
def env():
    from faspxx_b200 import capi, sol
    from oracle import oracle as O
    capi.init(0)
    O.build(ref=False)
    return capi, sol, O


def _solve(sol, alg, kw, A, b, x0, engine=None):
    s = sol.configure(alg, **kw)
    if engine is not None:
        s.SetPersistent(engine == "persistent")
        s.SetUseGraph(engine in ("graph", "graph_serial"))
        s.SetOverlapLaunch(engine != "graph_serial")
    s.Setup(sol.MAT(A))
    x = np.array(x0, dtype=np.float64, copy=True)
    code = s.Solve(b, x)
    return code, s.GetIterations(), s.GetNorm2(), x


def _check(name, got, port, cmpx):
    code, it, n2, x = got
    assert code == port.code, (name, code, port.code)
    assert it == port.iters, (name, it, port.iters)
    assert np.isnan(n2) == np.isnan(port.norm2), (name, n2, port.norm2)
    if cmpx:
        fin = np.isfinite(port.x)
        assert np.array_equal(np.isfinite(x), fin), name
        if fin.any():
            scale = max(np.max(np.abs(port.x[fin])), 1e-300)
            assert np.max(np.abs(x[fin] - port.x[fin])) <= 1e-12 * scale, name


@pytest.mark.parametrize("name", sorted(CASES))
def test_fault_outcome_matches_reference(env, name):
    capi, sol, O = env
    alg, kw, A, b, x0, cmpx = CASES[name]
    port = O.Solver("port", A, alg, **kw).solve(b, x0)
    _check(name, _solve(sol, alg, kw, A, b, x0), port, cmpx)


@pytest.mark.parametrize("engine", ["graph_serial", "plain", "persistent"])
@pytest.mark.parametrize("name", sorted(n for n in CASES if n.startswith("cg_")))
def test_cg_engines_on_faults(env, name, engine):
    capi, sol, O = env
    alg, kw, A, b, x0, cmpx = CASES[name]
    port = O.Solver("port", A, alg, **kw).solve(b, x0)
    _check(name, _solve(sol, alg, kw, A, b, x0, engine), port, cmpx)


@pytest.mark.parametrize("alg", ["cg", "bicgstab", "gmres"])
def test_mixed_precision_stops_on_nan(env, alg):
    capi, sol, O = env
    _, kw, A, b, x0, _ = CASES[f"{alg}_jac_nan_b"]
    modes = [capi.MIXED] + ([capi.MIXED_RELIABLE] if alg == "cg" else [])
    for mode in modes:
        s = sol.configure(alg, **kw)
        s.SetPrecision(mode, innerRelTol=1e-4, maxOuter=5)
        s.Setup(sol.MAT(A))
        x = np.zeros(A.nrow)
        code = s.Solve(b, x)
        assert code != 0 or np.isnan(s.GetNorm2()), (alg, mode, code)


def test_persistent_barrier_limit_expires_and_recovers(env):
    capi, sol, O = env
    from faspxx_b200 import problems as P
    A = P.poisson3d(24)
    b = A.matvec(P.seeded_uniform(A.nrow, 42))
    kw = dict(maxIter=500, minIter=0, relTol=1e-8, absTol=0.0, pcd="jacobi", pcdIter=1)
    s = sol.configure("cg", **kw)
    s.SetPersistent(True)
    s.Setup(sol.MAT(A))
    assert capi.lib.fasp_gpu_solver_set_barrier_limit(s.h, 1) == 0
    codes = []
    for _ in range(3):  # one poll: the first block to arrive cannot see 500+ others arrive
        try:
            codes.append(s.Solve(b, np.zeros(A.nrow)))
        except capi.FaspError as exc:
            codes.append(exc.code)
        if codes[-1] == capi.ERROR_CUDA:
            break
    assert codes[-1] == capi.ERROR_CUDA, codes
    assert capi.lib.fasp_gpu_solver_set_barrier_limit(s.h, 0) == 0
    x = np.zeros(A.nrow)
    assert s.Solve(b, x) == 0
    ref = O.solve("port", A, "cg", b, np.zeros(A.nrow), **kw)
    assert abs(s.GetIterations() - ref.iters) <= 1
    assert np.max(np.abs(x - ref.x)) <= 1e-6 * np.max(np.abs(ref.x))
