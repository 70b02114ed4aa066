"""MAT::Mult (src/MAT.cxx:715-800) on the CPU oracle against the reference's own products
(tests/golden/reference_mult.*): the restatement gives the same rows (columns in the
reference's first-appearance order, not sorted) and bit-identical values."""
import numpy as np
import pytest

from tests.golden import cases as G

CASES = G.mult_cases()


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    oracle.build(ref=False)
    return oracle


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference(O, name):
    L, R, want = CASES[name]
    got = O.mat_mult("port", L, R)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_products_are_unsorted_and_complete():
    """The fixtures exercise what the order rule is about: rows whose columns are not
    ascending, and values equal to a dense product."""
    unsorted = 0
    for L, R, (rp, ci, va) in CASES.values():
        dense = L.scipy().toarray() @ R.scipy().toarray() if hasattr(L, "scipy") else None
        for i in range(L.nrow):
            seg = ci[rp[i]:rp[i + 1]]
            unsorted += int(np.any(np.diff(seg.astype(np.int64)) < 0))
            assert len(np.unique(seg)) == len(seg)
        if dense is not None:
            C = np.zeros_like(dense)
            for i in range(L.nrow):
                C[i, ci[rp[i]:rp[i + 1]]] = va[rp[i]:rp[i + 1]]
            assert np.allclose(C, dense, rtol=1e-13, atol=1e-12)
    assert unsorted > 0


ADD = G.add_cases()


@pytest.mark.parametrize("name", sorted(ADD))
def test_add_restatement_matches_reference(O, name):
    a, A, b, B, want = ADD[name]
    code, got = O.mat_add("port", a, A, b, B)
    assert code == 0
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_add_fixture_repeats_an_appended_column():
    """repeated_appends: each row of B is [0, i+7, i+7, i+9, i+7]. Column 0 is appended first
    and takes the one extra slot MAT::Add searches besides A's entries, so the later repeats
    of column i+7 find no match and stay separate entries (sorted together)."""
    a, A, b, B, (rp, ci, va) = ADD["repeated_appends"]
    row = 20
    seg = ci[rp[row]:rp[row + 1]]
    assert np.count_nonzero(seg == row + 7) == 3 and np.count_nonzero(seg == 0) == 1
