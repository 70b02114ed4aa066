"""The CPU oracle (a C restatement of FASP++) pinned against the reference's own outputs.

The golden fixtures were produced by the reference compiled from its own sources
(tests/golden/make_golden.py). Solutions must agree bit for bit; residual histories agree
at the 6 significant digits the reference prints.
"""
import json
import os

import numpy as np
import pytest

from tests.golden import cases as G

GOLD = os.path.join(os.path.dirname(__file__), "golden")
RUNS = json.load(open(os.path.join(GOLD, "reference_runs.json")))
ARR = np.load(os.path.join(GOLD, "reference_runs.npz"))
CASES = {c["name"]: c for c in G.solver_cases()}


def hist_matches(port_hist, ref_hist):
    """Every value the reference printed equals the restatement's, rounded the same way."""
    for k, v in enumerate(ref_hist):
        if np.isnan(v):
            continue
        assert k < len(port_hist), k
        assert f"{port_hist[k]:.5e}" == f"{v:.5e}", (k, port_hist[k], v)


@pytest.mark.parametrize("name", sorted(CASES))
def test_port_matches_reference_run(oracle_built, name):
    O = oracle_built
    case = CASES[name]
    A, b, x0 = G.case_inputs(case)
    if case.get("store_b"):
        assert np.array_equal(b, ARR[name + "__b"])
    s = O.Solver("port", A, case["alg"], **case["kw"])
    for rep in range(case.get("repeat", 1)):
        key = name if rep == 0 else f"{name}__rep{rep}"
        r = s.solve(b, x0)
        meta = RUNS[key]
        assert r.code == meta["code"]
        assert r.iters == meta["iters"]
        assert r.norm2 == meta["norm2"]
        assert r.normInf == meta["normInf"]
        assert np.array_equal(r.x, ARR[key + "__x"])
        hist_matches(r.hist, ARR[key + "__hist"])


def test_spmv_known_answer(oracle_built):
    """utest/src/UnitTestsMAT.cxx:152-161: mat1 * 0.314 at 1e-14."""
    O = oracle_built
    A = G.small_csr(G.MAT1)
    y = O.spmv("port", A, np.array(G.MAT1["x"]))
    assert np.max(np.abs(y - np.array(G.MAT1["y"]))) < G.MAT1["tol"]


@pytest.mark.parametrize("d,w", [(G.JACOBI2, 1.0), (G.JACOBI2, 0.5), (G.JACOBI3, 1.0),
                                 (G.JACOBI3, 0.5)])
def test_jacobi_known_answer(oracle_built, d, w):
    """utest/src/UnitTestsJacobi.cxx: Jacobi and weighted Jacobi reach the octave solution."""
    O = oracle_built
    A = G.small_csr(d)
    r = O.solve("port", A, "jacobi", np.array(d["b"], float), np.zeros(A.nrow), maxIter=100,
                relTol=1e-9, weight=w)
    assert np.max(np.abs(r.x - np.array(d["xstar"]))) < d["tol"]


@pytest.mark.parametrize("name", [n for n, _ in G.transpose_cases()])
def test_transpose_matches_reference(oracle_built, name):
    O = oracle_built
    A = dict(G.transpose_cases())[name]
    z = np.load(os.path.join(GOLD, "reference_transpose.npz"))
    rp, ci, va, dp = O.transpose("port", A)
    assert np.array_equal(rp, z[name + "__rowPtr"])
    assert np.array_equal(ci, z[name + "__colInd"])
    assert np.array_equal(va, z[name + "__values"])
    assert np.array_equal(dp, z[name + "__diagPtr"])


def test_vec_reductions_follow_reference_order(oracle_built):
    """VEC::Dot/Norm2 sum in 4 interleaved partial sums (src/VEC.cxx:424-485)."""
    O = oracle_built
    rng = np.random.default_rng(3)
    for n in (0, 1, 3, 4, 5, 101, 1000):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        p = [0.0] * 4
        for i in range(n - n % 4):
            p[i % 4] += a[i] * b[i]
        for i in range(n - n % 4, n):
            p[0] += a[i] * b[i]
        assert O.dot("port", a, b) == ((p[0] + p[1]) + p[2]) + p[3]
        assert O.norminf("port", a) == (np.max(np.abs(a)) if n else 0.0)


def test_readmat_restatement_on_unsorted_rows():
    """SortCSRRow + CSRtoMAT: rows sorted by column, a zero diagonal inserted if missing."""
    import tempfile
    from faspxx_b200 import problems as P
    txt = "3\n1\n3\n4\n6\n2\n1\n3\n3\n1\n5.0\n2.0\n7.0\n1.0\n9.0\n"
    with tempfile.NamedTemporaryFile("w", suffix=".csr", delete=False) as f:
        f.write(txt)
    A = P.read_csr_text(f.name)
    os.unlink(f.name)
    assert A.rowPtr.tolist() == [0, 2, 4, 6]
    assert A.colInd.tolist() == [0, 1, 1, 2, 0, 2]
    assert A.values.tolist() == [2.0, 5.0, 0.0, 7.0, 9.0, 1.0]
