"""GPU parity: the CUDA library against the reference's recorded outputs and the CPU oracle.

Mirrors the reference's own unit tests (utest/src/UnitTestsMAT.cxx, UnitTestsJacobi.cxx,
UnitTestsVEC.cxx) and replays every golden solver run (tests/golden/cases.py) through the
C ABI. Tolerances, stated per check:

* SpMV / Residual: 1e-14 relative (sums are reordered, so not bit for bit);
* VEC reductions: 1e-13 relative;
* transpose (CSR -> CSC): bit-exact structure, order and values;
* solvers: the same return code, iteration count within +-1, the solution within
  1e-6 of the oracle's (relative to max(|x|, |x0|)); residual history entry k within
  max(1e-10, 10 x the case's sensitivity envelope up to entry k + 3) relative, plus the
  rounding floor of a residual norm (1e-15 of the initial residual). The envelope is the
  oracle (pinned bit for bit to the reference) rerun with every entry of b and x0 moved
  by one ulp: the GPU's reordered sums perturb each step by about that much, so where the
  reference reproduces itself the bar is 1e-10 over the whole history; entries past the
  point where the envelope reaches 1e-2 (the reference's own trajectories have
  decorrelated: chaotic BiCGStab) are not compared one by one. Cases whose
  stopping test sits at the rounding floor (FLOOR) or that the reference's own history
  shows to be erratic (ERRATIC) are held to the return code and a looser iteration window,
  stated below.
"""
import json
import os

import numpy as np
import pytest

from tests.golden import cases as G

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
RUNS = json.load(open(os.path.join(GOLD, "reference_runs.json")))
ARR = np.load(os.path.join(GOLD, "reference_runs.npz"))
CASES = {c["name"]: c for c in G.solver_cases()}

# stopping test at the rounding floor: relTol 1e-17 (see tests/golden/cases.py). The run
# ends in rounding noise: converged, ERROR_SOLVER_TOLSMALL after the false-convergence
# restarts, or (BiCGStab) the breakdown test |(ptmp, r0*)| <= 1e-40 between restarts
# (ERROR_DIVIDE_ZERO): the reference itself ends so for 14 of 40 one-ulp perturbations of
# b (after 65 to 317 iterations), TOLSMALL after 318-366 for the others.
FLOOR = {"fdm_cg_tolsmall": (0, -34), "fdm_bicgstab_tolsmall": (0, -34, -18)}
# BiCGStab on fem_small from x0 = 1, b = 0: the residual norm oscillates by orders of
# magnitude near the threshold; two reruns of the reference with reordered sums differ too
ERRATIC = {"fem_bicgstab": 3, "fem_bicgstab_jac": 3}


def perturbed(v, seed=1):
    """Every entry moved by one ulp, up or down (seeded)."""
    up = np.random.default_rng(seed).random(len(v)) < 0.5
    return np.where(up, np.nextafter(v, np.inf), np.nextafter(v, -np.inf))


def history_bound(h_ref, h_env):
    """Per-entry absolute bound: max(1e-10, 10 x running envelope 3 entries ahead) relative
    plus 1e-15 of the initial residual (the rounding floor of a residual norm)."""
    m = min(len(h_ref), len(h_env))
    env = np.zeros(len(h_ref))
    with np.errstate(invalid="ignore", divide="ignore"):
        env[:m] = np.nan_to_num(np.abs(h_env[:m] - h_ref[:m]) / h_ref[:m], nan=0.0)
    if m < len(h_ref):
        env[m:] = np.inf  # the perturbed run stopped earlier: no bar beyond it
    run = np.maximum.accumulate(env)
    ahead = np.minimum(np.arange(len(h_ref)) + 3, len(h_ref) - 1)
    bound = np.maximum(1e-10, 10.0 * np.minimum(run[ahead], 1.0)) * h_ref + 1e-15 * h_ref[0]
    # past 1e-2 the reference's own perturbed trajectory has decorrelated: not compared
    bound[run[ahead] >= 1e-2] = np.inf
    return bound


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


@pytest.fixture(scope="module")
def oracle():
    from oracle import oracle as O
    if not os.path.exists(O.PORT_SO):
        O.build(ref=False)
    return O


def test_spmv_known_answer(gpu):
    """utest/src/UnitTestsMAT.cxx:152-161 at TOL 1e-14."""
    A = G.small_csr(G.MAT1)
    M = gpu.MAT(A)
    x = gpu.DVec.from_numpy(np.array(G.MAT1["x"]))
    y = gpu.DVec(4)
    M.Apply(x, y)
    assert np.max(np.abs(y.numpy() - np.array(G.MAT1["y"]))) < G.MAT1["tol"]


def test_pattern_only_apply(gpu, oracle):
    """MAT::Apply on a sparsity structure treats every stored entry as 1 (MAT.cxx:420-451)."""
    A = G.matrix("fdm_10X10")
    P = type(A)(A.nrow, A.mcol, A.rowPtr, A.colInd, None)
    M = gpu.MAT(P)
    xv = np.random.default_rng(5).standard_normal(A.nrow)
    y = gpu.DVec(A.nrow)
    M.Apply(gpu.DVec.from_numpy(xv), y)
    ref = oracle.spmv("port", P, xv)
    assert np.max(np.abs(y.numpy() - ref)) <= 1e-14 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", ["fdm_10X10", "fem_small", "poisson3d_12", "convdiff_pe10",
                                  "vardiff_8"])
@pytest.mark.parametrize("lanes", [1, 2, 4, 8, 16, 32])
def test_spmv_matches_oracle(gpu, oracle, name, lanes):
    A = G.matrix(name)
    M = gpu.MAT(A)
    M.SetLanes(lanes)
    xv = np.random.default_rng(lanes).standard_normal(A.mcol)
    y = gpu.DVec(A.nrow)
    M.Apply(gpu.DVec.from_numpy(xv), y)
    ref = oracle.spmv("port", A, xv)
    assert np.max(np.abs(y.numpy() - ref)) <= 1e-14 * np.max(np.abs(ref))


def test_residual_and_shortcut(gpu, oracle):
    """MAT::Residual, including r = b when NormInf(x) < 1e-20 (MAT.cxx:459-462)."""
    A = G.matrix("fem_small")
    M = gpu.MAT(A)
    rng = np.random.default_rng(2)
    b = rng.standard_normal(A.nrow)
    for x in (rng.standard_normal(A.nrow), np.full(A.nrow, 1e-21)):
        r = gpu.DVec(A.nrow)
        M.Residual(gpu.DVec.from_numpy(b), gpu.DVec.from_numpy(x), r)
        ref = oracle.residual("port", A, b, x)
        assert np.max(np.abs(r.numpy() - ref)) <= 1e-14 * np.max(np.abs(ref))


def test_vec_operations(gpu, oracle):
    """utest/src/UnitTestsVEC.cxx: every VEC op against scalar loops."""
    rng = np.random.default_rng(4)
    for n in (1, 3, 100, 1000, 100003):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        da, db = gpu.DVec.from_numpy(a), gpu.DVec.from_numpy(b)
        assert abs(da.Dot(db) - oracle.dot("port", a, b)) <= 1e-13 * np.abs(a * b).sum()
        assert abs(da.Norm2() - oracle.norm2("port", a)) <= 1e-13 * oracle.norm2("port", a)
        assert da.NormInf() == oracle.norminf("port", a)
        da.AXPY(0.5, db)
        assert np.allclose(da.numpy(), a + 0.5 * b, rtol=1e-15, atol=0)
        da.set(a)
        da.XPAY(-2.0, db)
        assert np.allclose(da.numpy(), -2.0 * a + b, rtol=1e-15, atol=1e-15)
        da.set(a)
        da.AXPBY(3.0, -1.0, db)
        assert np.allclose(da.numpy(), 3.0 * a - b, rtol=1e-15, atol=1e-15)
        w = gpu.DVec(n)
        w.WAXPBY(2.0, da, 0.25, db)
        assert np.allclose(w.numpy(), 2.0 * (3.0 * a - b) + 0.25 * b, rtol=1e-14, atol=1e-14)
        w.Scale(-1.5)
        assert np.allclose(w.numpy(), -1.5 * (2.0 * (3.0 * a - b) + 0.25 * b), rtol=1e-14, atol=1e-14)


def test_reductions_are_deterministic(gpu):
    rng = np.random.default_rng(9)
    a = gpu.DVec.from_numpy(rng.standard_normal(5_000_003))
    vals = {a.Dot(a) for _ in range(5)}
    assert len(vals) == 1


@pytest.mark.parametrize("name", [n for n, _ in G.transpose_cases()])
def test_transpose_bit_exact(gpu, name):
    """CSR -> CSC in MAT::TransInPlace's exact order (MAT.cxx:479-538)."""
    A = dict(G.transpose_cases())[name]
    z = np.load(os.path.join(GOLD, "reference_transpose.npz"))
    T = gpu.MAT(A).Transpose()
    t = T.download()
    assert np.array_equal(t.rowPtr, z[name + "__rowPtr"])
    assert np.array_equal(t.colInd, z[name + "__colInd"])
    assert np.array_equal(t.values, z[name + "__values"])
    assert np.array_equal(T.diag_ptr(), z[name + "__diagPtr"])


def test_invalid_csr_is_rejected_before_upload(gpu):
    from faspxx_b200 import capi
    A = G.small_csr(G.MAT1)
    bad = type(A)(4, 4, A.rowPtr, A.colInd.copy(), A.values)
    bad.colInd[3] = 99
    with pytest.raises(capi.FaspError) as e:
        gpu.MAT(bad)
    assert e.value.code == -17


def _check_case(gpu, oracle, name, engine="graph", orth=None):
    case = CASES[name]
    A, b, x0 = G.case_inputs(case)
    M = gpu.MAT(A)
    s = gpu.configure(case["alg"], **case["kw"])
    if orth is not None:
        s.SetOrth(orth)
    s.SetPersistent(2 if engine == "cluster" else engine == "persistent")
    s.SetUseGraph(engine in ("graph", "graph_serial"))
    s.SetOverlapLaunch(engine != "graph_serial")
    s.Setup(M)
    po = oracle.Solver("port", A, case["alg"], **case["kw"])
    for rep in range(case.get("repeat", 1)):
        key = name if rep == 0 else f"{name}__rep{rep}"
        meta = RUNS[key]
        x = x0.copy()
        code = s.Solve(b, x)
        ref = po.solve(b, x0)
        assert ref.code == meta["code"] and ref.iters == meta["iters"]  # oracle pinned
        if name in FLOOR:
            assert code in FLOOR[name], (key, code)
        else:
            assert code == meta["code"], (key, code, meta["code"])
        it = s.GetIterations()
        if name in FLOOR:
            # the count of false-convergence restarts at the floor is chaotic: a converged or
            # TOLSMALL run must have reached the rounding floor; a breakdown may strike right
            # after a restart (the reference's own perturbed runs end so with true residuals
            # from 1e-14 to 0.15); the history is compared below up to where the
            # reference's own perturbed run decorrelates
            if code != -18:
                r = b - A.matvec(x)
                assert np.linalg.norm(r) <= 1e-13 * np.linalg.norm(b), key
        else:
            window = ERRATIC.get(name, 1)
            assert abs(it - meta["iters"]) <= window, (key, it, meta["iters"])
            scale = max(np.max(np.abs(ref.x)), np.max(np.abs(x0)), 1e-300)
            xtol = 1e-3 if name in ERRATIC else 1e-6
            assert np.max(np.abs(x - ref.x)) <= xtol * scale, key
        h = s.History()
        m = min(len(h), len(ref.hist))
        fin = np.isfinite(ref.hist[:m])
        assert np.array_equal(fin, np.isfinite(h[:m])), key
        if not fin.any():
            continue
        if rep > 0:
            continue  # repeated solves on one object: the first solve's envelope only
        # a fresh oracle object, so that state kept between solves (FGMRES's Z) is untouched
        env = oracle.Solver("port", A, case["alg"], **case["kw"]).solve(perturbed(b),
                                                                         perturbed(x0))
        bound = history_bound(ref.hist[:m], env.hist)
        dev = np.abs(h[:m] - ref.hist[:m])
        bad = np.nonzero(fin & (dev > bound))[0]
        assert len(bad) == 0, (key, int(bad[0]), float(dev[bad[0]] / ref.hist[bad[0]]))


@pytest.mark.parametrize("name", sorted(CASES))
def test_solver_parity(gpu, oracle, name):
    _check_case(gpu, oracle, name)


@pytest.mark.parametrize("engine", ["persistent", "cluster", "plain", "graph_serial"])
@pytest.mark.parametrize("name", ["fdm_pcg", "fem_pcg", "p2d_pcg", "p3d_cg", "vd_cg",
                                  "fdm_cg_min5", "fdm_cg_tolsmall"])
def test_cg_engines_match(gpu, oracle, name, engine):
    """The device-driven CG meets the same bars run as CUDA graphs of its two kernels with
    overlapped launches (the default, exercised by test_solver_parity), as graphs with
    ordinary launches, as one persistent cooperative kernel, as one persistent thread-block
    cluster, and as plain launches."""
    _check_case(gpu, oracle, name, engine=engine)


@pytest.mark.parametrize("prec", ["FP64", "MIXED_RELIABLE"])
def test_cluster_engine_small_system(gpu, prec):
    """The one-cluster persistent CG (16 blocks meeting at the hardware cluster barrier) on a
    2D Poisson system, FP64 and FP32 iterations with reliable updates: the default engine's
    code and iteration count, the tolerance on the true residual."""
    from faspxx_b200 import capi, problems as P
    A = P.poisson2d(128)
    b = A.matvec(P.seeded_uniform(A.nrow, 42))
    out = []
    for mode in (0, 2):
        s = gpu.configure("cg", maxIter=2000, relTol=1e-8, absTol=0.0, pcd="jacobi",
                          pcdWeight=1.0, pcdIter=1)
        if prec != "FP64":
            s.SetPrecision(getattr(capi, prec), innerRelTol=1e-2)
        s.SetPersistent(mode)
        s.Setup(gpu.MAT(A))
        x = np.zeros(A.nrow)
        out.append((s.Solve(b, x), s.GetIterations(), x))
    (c0, i0, _), (c2, i2, x2) = out
    assert c0 == c2 == 0 and abs(i0 - i2) <= 1, (i0, i2)
    assert np.linalg.norm(b - A.matvec(x2)) <= 1e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("name", sorted(n for n in CASES if CASES[n]["alg"] in ("gmres",
                                                                                  "fgmres")))
def test_gmres_cgs2_parity(gpu, oracle, name):
    """GMRES with classical Gram-Schmidt reorthogonalised in the same step (CGS2, three passes
    over the basis) meets the bars of the default delayed variant (DCGS2, checked by
    test_solver_parity) against the reference's modified Gram-Schmidt: code, iteration
    count, solution and the residual history within the reference's own one-ulp envelope."""
    from faspxx_b200 import capi
    _check_case(gpu, oracle, name, orth=capi.ORTH_CGS2)


def test_known_answer_jacobi(gpu):
    """utest/src/UnitTestsJacobi.cxx: x* of the octave solutions at 1e-5."""
    for d in (G.JACOBI2, G.JACOBI3):
        for w in (1.0, 0.5):
            A = G.small_csr(d)
            s = gpu.configure("jacobi", maxIter=100, relTol=1e-9, weight=w)
            s.Setup(gpu.MAT(A))
            x = np.zeros(A.nrow)
            s.Solve(np.array(d["b"], float), x)
            assert np.max(np.abs(x - np.array(d["xstar"]))) < d["tol"]


def test_mgs_orthogonalisation_matches_reference_ops(gpu, oracle):
    """GMRES with the reference's modified Gram-Schmidt op sequence."""
    from faspxx_b200 import capi
    for name in ("fem_gmres_jac", "cd_pe10_gmres", "fem_fgmres_jac2"):
        case = CASES[name]
        A, b, x0 = G.case_inputs(case)
        s = gpu.configure(case["alg"], **case["kw"])
        s.SetOrth(capi.ORTH_MGS)
        s.Setup(gpu.MAT(A))
        x = x0.copy()
        assert s.Solve(b, x) == RUNS[name]["code"]
        assert abs(s.GetIterations() - RUNS[name]["iters"]) <= 1
        ref = oracle.solve("port", A, case["alg"], b, x0, **case["kw"])
        scale = max(np.max(np.abs(ref.x)), np.max(np.abs(x0)))
        assert np.max(np.abs(x - ref.x)) <= 1e-6 * scale


def test_clean_resets_fgmres_basis(gpu, oracle):
    """FGMRES keeps Z between solves (FGMRES.cxx:158-159) until Clean() (FGMRES.cxx:83-105)."""
    case = CASES["fem_fgmres_jac2"]
    A, b, x0 = G.case_inputs(case)
    s = gpu.configure(case["alg"], **case["kw"])
    s.Setup(gpu.MAT(A))
    x = x0.copy()
    s.Solve(b, x)
    s.Clean()
    x = x0.copy()
    s.Solve(b, x)
    assert abs(s.GetIterations() - RUNS["fem_fgmres_jac2"]["iters"]) <= 1
