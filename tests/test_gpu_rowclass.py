"""Row-class storage of constant-coefficient matrices: the thread-per-row SpMV reads a 2-byte
class id per row from a table of (column offset, value) lists instead of the CSR arrays.

Bar: bit-exact. Both forms accumulate each row's entries in CSR order with one FMA per
entry, so MAT::Apply, MAT::Residual and whole solves (iteration counts, solutions and
residual histories) are identical with the form on and off.
"""
import numpy as np
import pytest

from faspxx_b200 import problems as P
from tests.golden import cases as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


def _stencils():
    return {
        "poisson2d_40": P.poisson2d(40),
        "poisson3d_20": P.poisson3d(20),
        "convdiff3d_16_pe10": P.convdiff3d(16, 10.0),
        "fdm_10X10": G.matrix("fdm_10X10"),
    }


@pytest.mark.parametrize("name", list(_stencils()))
def test_apply_and_residual_bit_exact(gpu, name):
    A = _stencils()[name]
    M = gpu.MAT(A)
    on, classes, entries = M.RowClassInfo()
    assert on and 0 < classes <= 4096 and entries <= max(64, A.nnz // 8)
    rng = np.random.default_rng(1)
    x = gpu.DVec.from_numpy(rng.standard_normal(A.mcol))
    b = gpu.DVec.from_numpy(rng.standard_normal(A.nrow))
    y_rc, r_rc = gpu.DVec(A.nrow), gpu.DVec(A.nrow)
    M.Apply(x, y_rc)
    M.Residual(b, x, r_rc)
    M.SetRowClass(False)
    assert not M.RowClassInfo()[0]
    y, r = gpu.DVec(A.nrow), gpu.DVec(A.nrow)
    M.Apply(x, y)
    M.Residual(b, x, r)
    assert np.array_equal(y_rc.numpy(), y.numpy())
    assert np.array_equal(r_rc.numpy(), r.numpy())
    # and both agree with the host product to rounding
    ref = A.matvec(x.numpy())
    assert np.max(np.abs(y.numpy() - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_variable_coefficients_stay_csr(gpu):
    kappa = 10.0 ** np.random.default_rng(2).uniform(-1, 1, 12 ** 3)
    M = gpu.MAT(P.vardiff3d(12, kappa))
    assert M.RowClassInfo() == (False, 0, 0)
    M.SetRowClass(True)  # nothing to switch on
    assert M.RowClassInfo()[0] is False


@pytest.mark.parametrize("alg,prec", [("cg", "FP64"), ("cg", "MIXED_RELIABLE"),
                                      ("bicgstab", "FP64"), ("gmres", "FP64"),
                                      ("fgmres", "MIXED")])
def test_solves_identical_with_and_without_row_classes(gpu, alg, prec):
    from faspxx_b200 import capi
    A = P.convdiff3d(14, 0.1) if alg != "cg" else P.poisson3d(18)
    b = A.matvec(np.random.default_rng(4).uniform(-1, 1, A.nrow))
    out = []
    for rc in (True, False):
        M = gpu.MAT(A)
        M.SetRowClass(rc)
        s = gpu.configure(alg, maxIter=2000, relTol=1e-9, absTol=0.0, pcd="jacobi",
                          pcdWeight=2.0 / 3.0 if alg != "cg" else 1.0, pcdIter=1)
        if prec != "FP64":
            s.SetPrecision(getattr(capi, prec))
        s.Setup(M)
        x = np.zeros(A.nrow)
        code = s.Solve(b, x)
        out.append((code, s.GetIterations(), x, s.History()))
    (c1, i1, x1, h1), (c2, i2, x2, h2) = out
    assert c1 == c2 == 0 and i1 == i2
    assert np.array_equal(x1, x2)
    assert np.array_equal(np.nan_to_num(h1), np.nan_to_num(h2))
