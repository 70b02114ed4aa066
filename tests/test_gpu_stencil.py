"""Matrix-free grid operators on the GPU (fasp_gpu_mat_create_stencil): the counterpart of
the reference's matrix-free LOP example (example/TestMatFree.cxx:26-176).

Bar: a grid operator computes exactly what the assembled CSR matrix computes. Its rows are
grid points in x-fastest order and its entries the stencil points inside the grid in
ascending column order, so Apply, Residual, transposes and whole solves (iteration counts,
solutions and residual histories) are bit-identical to those of MAT(csr) of the same
matrix, in every solver and precision. Against the reference itself: the matrix-free
example's CG runs (tests/golden/reference_matfree.json) -- same iteration counts (+-1, the
GPU's reduction order differs), residual norms and L2 errors.
"""
import json
import os

import numpy as np
import pytest

from faspxx_b200 import problems as P

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                   "reference_matfree.json")))

FIVE = [((0, -1), -1.0), ((-1, 0), -1.0), ((0, 0), 4.0), ((1, 0), -1.0), ((0, 1), -1.0)]
SEVEN = [((0, 0, -1), -1.0), ((0, -1, 0), -1.0), ((-1, 0, 0), -1.0), ((0, 0, 0), 6.0),
         ((1, 0, 0), -1.0), ((0, 1, 0), -1.0), ((0, 0, 1), -1.0)]


def _convdiff7(N, peclet):
    """The upwind convection-diffusion stencil of problems.convdiff3d as grid points."""
    A = P.convdiff3d(N, peclet)
    n2 = N * N
    # an interior row has all seven entries; read their coefficients off the CSR matrix
    row = N // 2 + N * (N // 2) + n2 * (N // 2)
    b, e = A.rowPtr[row], A.rowPtr[row + 1]
    pts = []
    for k in range(b, e):
        d = int(A.colInd[k]) - row
        off = {-n2: (0, 0, -1), -N: (0, -1, 0), -1: (-1, 0, 0), 0: (0, 0, 0), 1: (1, 0, 0),
               N: (0, 1, 0), n2: (0, 0, 1)}[d]
        pts.append((off, float(A.values[k])))
    return A, pts


CASES = {
    "poisson2d_33x20": ((33, 20), FIVE),
    "poisson3d_12": ((12, 12, 12), SEVEN),
    "poisson3d_9x5x7": ((9, 5, 7), SEVEN),
    "line_reach3_40": ((40,), [((-3,), 0.25), ((-2,), -0.5), ((-1,), -1.0), ((0,), 4.5),
                               ((1,), -1.25), ((2,), -0.5), ((3,), 0.125)]),
    "nine_point_15x11": ((15, 11), [((dx, dy), 8.0 if dx == dy == 0 else -1.0 - 0.1 * dx)
                                    for dy in (-1, 0, 1) for dx in (-1, 0, 1)]),
    "tiny_2x1x3": ((2, 1, 3), SEVEN),
    "no_diagonal_7": ((7, 6), [((0, -1), 1.0), ((-1, 0), 2.0), ((1, 0), -3.0)]),
}


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


def _pair(gpu, name):
    shape, pts = CASES[name]
    G = gpu.MAT.Stencil(shape, pts)
    csr = G.download()
    return G, csr, gpu.MAT(csr)


def _assembled(shape, pts):
    """The CSR matrix of a grid stencil, assembled here point by point."""
    dims = list(shape) + [1] * (3 - len(shape))
    nx, ny, nz = dims
    offs = sorted(((tuple(list(o) + [0] * (3 - len(o))), c) for o, c in pts),
                  key=lambda t: t[0][0] + nx * (t[0][1] + ny * t[0][2]))
    rp, ci, va = [0], [], []
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                row = ix + nx * (iy + ny * iz)
                for (dx, dy, dz), c in offs:
                    jx, jy, jz = ix + dx, iy + dy, iz + dz
                    if 0 <= jx < nx and 0 <= jy < ny and 0 <= jz < nz:
                        ci.append(row + dx + nx * (dy + ny * dz))
                        va.append(c)
                rp.append(len(ci))
    n = nx * ny * nz
    return P.CSRMatrix(n, n, np.array(rp, np.uint32), np.array(ci, np.uint32),
                       np.array(va, np.float64))


@pytest.mark.parametrize("name", sorted(CASES))
def test_download_is_the_assembled_matrix(gpu, name):
    shape, pts = CASES[name]
    G = gpu.MAT.Stencil(shape, pts)
    A = _assembled(shape, pts)
    D = G.download()
    assert (G.GetRowSize(), G.GetNNZ()) == (A.nrow, A.nnz)
    for got, want in zip((D.rowPtr, D.colInd, D.values), (A.rowPtr, A.colInd, A.values)):
        assert np.array_equal(got, want)
    assert G.RowClassInfo()[0] == 3


def test_stencil_of_the_generators():
    """The grid stencils used below are the library's own test matrices."""
    A = _assembled((12, 12, 12), SEVEN)
    B = P.poisson3d(12)
    assert np.array_equal(A.rowPtr, B.rowPtr) and np.array_equal(A.colInd, B.colInd)
    assert np.array_equal(A.values, B.values)
    C, pts = _convdiff7(10, 10.0)
    D = _assembled((10, 10, 10), pts)
    assert np.array_equal(C.colInd, D.colInd) and np.array_equal(C.values, D.values)


@pytest.mark.parametrize("name", sorted(CASES))
def test_apply_and_residual_bit_exact(gpu, name):
    G, csr, M = _pair(gpu, name)
    rng = np.random.default_rng(3)
    x = gpu.DVec.from_numpy(rng.standard_normal(csr.nrow))
    b = gpu.DVec.from_numpy(rng.standard_normal(csr.nrow))
    out = []
    for op in (G, M):
        y, r = gpu.DVec(csr.nrow), gpu.DVec(csr.nrow)
        op.Apply(x, y)
        op.Residual(b, x, r)
        out.append((y.numpy(), r.numpy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_transpose_is_the_negated_stencil(gpu):
    A, pts = _convdiff7(9, 10.0)
    G = gpu.MAT.Stencil((9, 9, 9), pts)
    T = G.Transpose()
    assert T.RowClassInfo()[0] == 3
    Tc = gpu.MAT(A).Transpose().download()
    D = T.download()
    for got, want in zip((D.rowPtr, D.colInd, D.values), (Tc.rowPtr, Tc.colInd, Tc.values)):
        assert np.array_equal(got, want)


@pytest.mark.parametrize("alg,prec", [("cg", "FP64"), ("cg", "MIXED_RELIABLE"),
                                      ("cg", "MIXED"), ("bicgstab", "FP64"),
                                      ("gmres", "FP64"), ("fgmres", "MIXED"),
                                      ("jacobi", "FP64"), ("mg", "FP64")])
def test_solves_identical_to_csr(gpu, alg, prec):
    from faspxx_b200 import capi
    if alg in ("cg", "jacobi", "mg"):
        shape, pts, A = (14, 13, 12), SEVEN, None
    else:
        A, pts = _convdiff7(12, 0.1)
        shape = (12, 12, 12)
    G = gpu.MAT.Stencil(shape, pts)
    M = gpu.MAT(G.download())
    n = G.GetRowSize()
    b = M.download().matvec(np.random.default_rng(4).uniform(-1, 1, n))
    out = []
    for op in (G, M):
        kw = dict(maxIter=3000 if alg != "jacobi" else 400, relTol=1e-9, absTol=0.0)
        if alg not in ("jacobi", "mg"):
            kw.update(pcd="jacobi", pcdWeight=2.0 / 3.0 if alg != "cg" else 1.0, pcdIter=1)
        if alg == "jacobi":
            kw.update(weight=2.0 / 3.0)
        s = gpu.configure(alg, **kw)
        if prec != "FP64":
            s.SetPrecision(getattr(capi, prec))
        s.Setup(op)
        x = np.zeros(n)
        code = s.Solve(b, x)
        out.append((code, s.GetIterations(), x, np.nan_to_num(s.History())))
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][3], out[1][3])


def _l2_error(dim, x):
    h = 1.0 / dim
    k = np.arange(1, dim)
    u = np.outer(np.sin(np.pi * k * h), np.sin(np.pi * k * h)).ravel()
    return float(np.sqrt(np.sum((x - u) ** 2) * h * h))


@pytest.mark.parametrize("dim", [16, 32, 64, 128, 256, 512])
def test_reference_matrix_free_example(gpu, dim):
    """TestMatFree.cxx:178-255 on the GPU grid operator: CG without preconditioner,
    maxIter 10000, restart 20, absTol 1e-12, relTol 1e-8, x0 = 0.25, the example's
    right-hand side; second-order convergence of the L2 error."""
    from oracle import oracle as O
    ref = GOLD[str(dim)]
    G = gpu.MAT.Stencil((dim - 1, dim - 1), FIVE)
    s = gpu.configure("cg", maxIter=10000, restart=20, relTol=1e-8, absTol=1e-12)
    s.Setup(G)
    x = np.full(G.GetRowSize(), 0.25)
    assert s.Solve(O.matfree_rhs(dim), x) == 0
    assert abs(s.GetIterations() - ref["iters"]) <= 1
    assert abs(s.GetNorm2() - float(ref["norm2"])) <= 0.05 * float(ref["norm2"])
    # the printed error has 5 significant digits
    assert abs(_l2_error(dim, x) - float(ref["l2err"])) <= 1e-4 * float(ref["l2err"])


@pytest.mark.parametrize("bad", ["reach4", "duplicate", "too_many", "empty_grid",
                                 "sampled_outer", "lanes"])
def test_rejections(gpu, bad):
    from faspxx_b200 import capi
    with pytest.raises(capi.FaspError) as e:
        if bad == "reach4":
            gpu.MAT.Stencil((20,), [((4,), 1.0), ((0,), 2.0)])
        elif bad == "duplicate":
            gpu.MAT.Stencil((20,), [((1,), 1.0), ((1,), 2.0)])
        elif bad == "too_many":
            gpu.MAT.Stencil((9, 9), [((dx, dy), 1.0) for dx in (-2, -1, 0, 1, 2)
                                     for dy in (-1, 0, 1, 2)])
        elif bad == "empty_grid":
            gpu.MAT.Stencil((0, 4), FIVE)
        elif bad == "sampled_outer":
            G = gpu.MAT.Stencil((6, 6), FIVE)
            v = gpu.DVec.from_numpy(np.ones(36))
            G.SampledOuter(v, v, 1.0, gpu.DVec(G.GetNNZ()))
        else:
            gpu.MAT.Stencil((6, 6), FIVE).SetLanes(4)
    assert e.value.code in (-12, -15)
