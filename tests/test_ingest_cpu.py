"""ReadMat's conversions on the CPU: the oracle's restatement of MTXtoMAT and of the .csr
branch (ReadCSR's shift, SortCSRRow, CSRtoMAT) against the reference's own results
(tests/golden/reference_ingest.*, written by make_golden.py from the compiled reference),
and the host-side text readers. Bar: bit-exact arrays and the same return code."""
import os

import numpy as np
import pytest

from faspxx_b200 import problems as P
from tests.golden import cases as G

CASES = G.ingest_cases()


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    oracle.build(ref=False)
    return oracle


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference(O, name):
    c = CASES[name]
    a, b, v = c["inputs"]
    if c["kind"] == "mtx":
        code, res = O.mtx_to_mat("port", c["nrow"], c["mcol"], a, b, v)
    else:
        code, res = O.csr_to_mat("port", c["nrow"], a, b, v)
    assert code == c["code"]
    if c["expected"] is None:
        assert res is None
        return
    for got, want in zip(res, c["expected"]):
        assert got.dtype == want.dtype and np.array_equal(got, want)


def test_cases_cover_the_edge_cases():
    """The fixtures hold what the conversions must get right: 1-based unsorted files,
    duplicates, missing and empty-row diagonals, long rows of every sort class, and the
    inputs the reference leaves empty."""
    def dup_and_missing(c):
        rp, ci, _ = c["expected"]
        rows = np.repeat(np.arange(c["nrow"]), np.diff(rp.astype(np.int64)))
        dup = np.any((np.diff(ci.astype(np.int64)) == 0) & (np.diff(rows) == 0))
        return dup
    assert dup_and_missing(CASES["random_dup_mtx"]) and dup_and_missing(CASES["dup1_csr"])
    assert CASES["fem_small_csr"]["inputs"][0][0] == 1  # 1-based file
    lens = np.diff(CASES["long_rows_mtx"]["expected"][0].astype(np.int64))
    assert lens.max() > 8192 and ((lens > 32) & (lens <= 4096)).any() and (lens <= 8).any()
    assert CASES["tall_mtx"]["expected"] is None and CASES["badcol_mtx"]["expected"] is None
    # empty rows (other than row 0) in the input become a lone zero diagonal
    rp, ci, va = CASES["random_dup_mtx"]["expected"]
    ri = CASES["random_dup_mtx"]["inputs"][0]
    empty = np.setdiff1d(np.arange(60), ri)
    assert len(empty) and all(rp[i + 1] - rp[i] == 1 and ci[rp[i]] == i and va[rp[i]] == 0.0
                              for i in empty)


def test_text_readers_round_trip(tmp_path):
    c = CASES["random_dup_mtx"]
    p = str(tmp_path / "m.mtx")
    G.write_mtx(p, c["nrow"], c["mcol"], *c["inputs"])
    nrow, mcol, ri, ci, va = P.read_mtx_raw(p)
    assert (nrow, mcol) == (c["nrow"], c["mcol"])
    for got, want in zip((ri, ci, va), c["inputs"]):
        assert np.array_equal(got, want)
    c = CASES["fdm_10X10_csr"]
    p = str(tmp_path / "m.csr")
    G.write_csr(p, c["nrow"], *c["inputs"])
    n, rp, ci, va = P.read_csr_raw(p)
    for got, want in zip((rp, ci, va), c["inputs"]):
        assert np.array_equal(got, want)
    A = P.read_csr_text(p)  # the host restatement used by the solver fixtures
    for got, want in zip((A.rowPtr, A.colInd, A.values), c["expected"]):
        assert np.array_equal(got, want)


def test_restatement_rejects_what_the_reference_cannot_index(O):
    # a row index beyond nrow: the reference's MTXtoCSR writes out of bounds
    code, res = O.mtx_to_mat("port", 3, 3, [0, 3], [0, 1], [1.0, 2.0])
    assert code == -17 and res is None
    # rowPtr starting at 2: neither 0- nor 1-based
    code, res = O.csr_to_mat("port", 2, [2, 3, 4], [0, 1], [1.0, 2.0])
    assert code == -17 and res is None
