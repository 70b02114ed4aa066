"""MG with transfer operators on the GPU (fasp_gpu_solver_set_mg_transfer).

The reference's MG cycle (MG.cxx:105-152) with per-level operators and separate restriction
and prolongation has no counterpart the reference can run (its SetupLevel stores one operator
for both transfers and every residual uses the top-level matrix), so the oracle restates the
same cycle (orc_mg_set_level) with the operators the GPU uses: restrictions that are P's exact
transpose (MAT::TransInPlace) and Galerkin coarse operators R (A P) from MAT::Mult -- both
bit-identical on the two sides. Bar, as for the other solvers: the same return code and
iteration count, residual histories within 1e-9 relative (1e-6 where the residual is within
1e-6 of the first, near the rounding level), solutions within 1e-9 relative.
Plus what makes it multigrid: geometric V-cycles reduce the residual by a grid-independent
factor (<= 0.25 per cycle here).
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


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    return oracle


def _interp1d(nf):
    nc = (nf - 1) // 2
    rows = []
    for i in range(nf):
        if i % 2 == 1:
            rows.append([((i - 1) // 2, 1.0)])
        else:
            r = []
            if i // 2 - 1 >= 0:
                r.append((i // 2 - 1, 0.5))
            if i // 2 < nc:
                r.append((i // 2, 0.5))
            rows.append(r)
    return rows, nc


def _interp(nf, dim):
    """Linear (2D: bilinear, 3D: trilinear) prolongation from the (nf-1)/2 grid, x fastest."""
    r1, nc = _interp1d(nf)
    rp, ci, va = [0], [], []
    idx = np.indices((nf,) * dim).reshape(dim, -1).T[:, ::-1]  # x fastest
    for pt in idx:
        terms = [(0, 1.0)]
        for d in range(dim):
            terms = [(c + (nc ** d) * cc, w * ww) for (c, w) in terms for (cc, ww) in r1[pt[d]]]
        for c, w in terms:
            ci.append(c)
            va.append(w)
        rp.append(len(ci))
    return P.CSRMatrix(nf ** dim, nc ** dim, np.array(rp, np.uint32), np.array(ci, np.uint32),
                       np.array(va, np.float64))


def _hierarchy(O, A, nf, dim, levels):
    out, Al = [], A
    for _ in range(levels):
        Pm = _interp(nf, dim)
        R = P.CSRMatrix(Pm.mcol, Pm.nrow, *O.transpose("port", Pm)[:3])
        AP = P.CSRMatrix(Al.nrow, Pm.mcol, *O.mat_mult("port", Al, Pm))
        Ac = P.CSRMatrix(Pm.mcol, Pm.mcol, *O.mat_mult("port", R, AP))
        out.append((Pm, R, Ac))
        Al, nf = Ac, (nf - 1) // 2
    return out


KW = dict(maxIter=60, relTol=1e-9, absTol=0.0, mgCycles=1,
          mgSmooth=dict(maxIter=2, minIter=2, weight=2.0 / 3.0),
          mgCoarse=dict(maxIter=40, minIter=40, weight=2.0 / 3.0))


def _gpu_mg(gpu, M, levels, explicit, **kw):
    s = gpu.configure("mg", mgLevels=len(levels), **{**KW, **kw})
    keep = []
    for l, (Pm, R, Ac) in enumerate(levels):
        gP = gpu.MAT(Pm)
        gR = gpu.MAT(R) if explicit else None
        gA = gpu.MAT(Ac) if explicit else None
        keep += [gP, gR, gA]
        s.SetTransfer(l, gP, gR, gA)
    s.Setup(M)
    s._keep = keep
    return s


@pytest.mark.parametrize("case", ["2d_31_3levels_galerkin", "2d_31_3levels_explicit",
                                  "3d_15_2levels_galerkin", "2d_31_wcycle"])
def test_matches_oracle(gpu, O, case):
    dim = 3 if case.startswith("3d") else 2
    nf = 15 if dim == 3 else 31
    L = 2 if "2levels" in case else 3
    A = P.poisson3d(nf) if dim == 3 else P.poisson2d(nf)
    levels = _hierarchy(O, A, nf, dim, L)
    extra = dict(mgCycles=2) if "wcycle" in case else {}
    b = A.matvec(np.random.default_rng(8).uniform(-1, 1, A.nrow))
    ref = O.Solver("port", A, "mg", mgLevels=L, **{**KW, **extra})
    for l, (Pm, R, Ac) in enumerate(levels):
        ref.set_mg_level(l, Pm, R, Ac)
    r = ref.solve(b, np.zeros(A.nrow))
    s = _gpu_mg(gpu, gpu.MAT(A), levels, "explicit" in case, **extra)
    x = np.zeros(A.nrow)
    code = s.Solve(b, x)
    assert code == r.code and s.GetIterations() == r.iters
    h = s.History()[: r.iters + 1]
    # residuals well above the rounding level agree to 1e-9; near it (the last cycles, where
    # b - A x cancels to 1e-9 of b) to 1e-6
    big = r.hist > 1e-6 * r.hist[0]
    assert np.allclose(h[big], r.hist[big], rtol=1e-9, atol=0.0)
    assert np.allclose(h, r.hist, rtol=1e-6, atol=0.0)
    assert np.max(np.abs(x - r.x)) <= 1e-9 * np.max(np.abs(r.x))
    assert r.iters <= 20  # it is multigrid: a few V-cycles reach 1e-9


@pytest.mark.parametrize("nf", [31, 63, 127])
def test_grid_independent_convergence(gpu, O, nf):
    """Galerkin V(2,2) cycles on 2D Poisson down to a 3 x 3 coarsest grid (40 Jacobi sweeps
    solve it): the residual falls by at most 0.25 per cycle at every size (the GPU forms R
    and the coarse operators itself)."""
    A = P.poisson2d(nf)
    L = int(np.log2((nf + 1) // 4))
    levels = _hierarchy(O, A, nf, 2, L)
    s = _gpu_mg(gpu, gpu.MAT(A), levels, False)
    b = A.matvec(np.random.default_rng(2).uniform(0, 1, A.nrow))
    x = np.zeros(A.nrow)
    assert s.Solve(b, x) == 0
    h = s.History()[: s.GetIterations() + 1]
    rates = h[2:] / h[1:-1]
    assert np.max(rates) <= 0.25, rates
    assert np.linalg.norm(b - A.matvec(x)) <= 1e-9 * np.linalg.norm(b) * 1.01


def test_grid_operator_with_given_coarse_operators(gpu, O):
    """A matrix-free fine level (no stored values, so no Galerkin product) with the coarse
    operators given: same iterations as the stored matrix."""
    nf = 31
    A = P.poisson2d(nf)
    levels = _hierarchy(O, A, nf, 2, 2)
    five = [((0, -1), -1.0), ((-1, 0), -1.0), ((0, 0), 4.0), ((1, 0), -1.0), ((0, 1), -1.0)]
    G = gpu.MAT.Stencil((nf, nf), five)
    b = A.matvec(np.random.default_rng(5).uniform(0, 1, A.nrow))
    out = []
    for M in (G, gpu.MAT(A)):
        s = _gpu_mg(gpu, M, levels, True)
        x = np.zeros(A.nrow)
        assert s.Solve(b, x) == 0
        out.append((s.GetIterations(), x))
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])


def test_setup_errors(gpu, O):
    from faspxx_b200 import capi
    A = P.poisson2d(15)
    levels = _hierarchy(O, A, 15, 2, 2)
    s = gpu.configure("mg", mgLevels=3, maxIter=5)
    Pm = gpu.MAT(levels[0][0])
    s.SetTransfer(0, Pm)
    with pytest.raises(capi.FaspError) as e:  # levels 1 and 2 missing
        s.Setup(gpu.MAT(A))
    assert e.value.code == -12
    s = gpu.configure("mg", mgLevels=1, maxIter=5)
    s.SetTransfer(0, gpu.MAT(levels[1][0]))  # the 7x7 -> 3x3 prolongation on a 15x15 grid
    with pytest.raises(capi.FaspError) as e:
        s.Setup(gpu.MAT(A))
    assert e.value.code == -16


# ---- MG as a preconditioner (SOL::SetupPCD with an MG object) -----------------------------

PKW = dict(mgCycles=1, mgSmooth=dict(maxIter=2, minIter=2, weight=2.0 / 3.0),
           mgCoarse=dict(maxIter=40, minIter=40, weight=2.0 / 3.0))


@pytest.mark.parametrize("alg,transfers", [("cg", True), ("gmres", True), ("cg", False),
                                           ("bicgstab", True)])
def test_mg_preconditioned_krylov_matches_oracle(gpu, O, alg, transfers):
    """One V-cycle from zero as the preconditioner (MG::Solve with minIter = maxIter = 1):
    Galerkin transfers (or the reference's identity transfers), same bar as the solvers."""
    nf = 63
    A = P.poisson2d(nf) if alg == "cg" else P.convdiff3d(15, 0.1)
    dim = 2 if alg == "cg" else 3
    nf = nf if alg == "cg" else 15
    L = 4 if alg == "cg" else 2
    levels = _hierarchy(O, A, nf, dim, L) if transfers else []
    kw = dict(maxIter=300, relTol=1e-10, absTol=0.0, pcd="mg", pcdIter=1, mgLevels=L, **PKW)
    if alg != "cg":
        kw.update(restart=30, maxRestart=30, minRestart=30) if alg == "gmres" else None
    b = A.matvec(np.random.default_rng(6).uniform(-1, 1, A.nrow))
    ref = O.Solver("port", A, alg, **kw)
    for l, (Pm, R, Ac) in enumerate(levels):
        ref.set_mg_level(l, Pm, R, Ac)
    r = ref.solve(b, np.zeros(A.nrow))
    s = gpu.configure(alg, **kw)
    keep = []
    for l, (Pm, R, Ac) in enumerate(levels):
        gP = gpu.MAT(Pm)
        keep.append(gP)
        s.transfers = getattr(s, "transfers", {})
        s.transfers[l] = (gP, None, None)
    s.Setup(gpu.MAT(A))
    x = np.zeros(A.nrow)
    code = s.Solve(b, x)
    if alg == "bicgstab":
        # the reference's BiCGStab applies the preconditioner to A p and A s separately
        # (BiCGStab.cxx:116-139); with a preconditioner that does not commute with A the
        # iteration is erratic and rounding-sensitive, so the bar is the outcome: both
        # converge, in counts within 15%, to the tolerance
        assert code == r.code == 0 and abs(s.GetIterations() - r.iters) <= 0.15 * r.iters
        assert np.linalg.norm(b - A.matvec(x)) <= 1e-9 * np.linalg.norm(b)
        return
    assert code == r.code and abs(s.GetIterations() - r.iters) <= 1
    n = min(s.GetIterations(), r.iters)
    h = s.History()[: n + 1]
    big = r.hist[: n + 1] > 1e-6 * r.hist[0]
    assert np.allclose(h[big], r.hist[: n + 1][big], rtol=1e-8, atol=0.0)
    assert np.max(np.abs(x - r.x)) <= 1e-8 * np.max(np.abs(r.x))
    if transfers and alg == "cg":
        assert r.iters <= 12  # against ~200 with Jacobi on this grid


def test_mg_preconditioner_rejects_mixed_precision(gpu):
    from faspxx_b200 import capi
    s = gpu.configure("cg", maxIter=10, pcd="mg", pcdIter=1, mgLevels=1)
    s.SetPrecision(capi.MIXED)
    with pytest.raises(capi.FaspError) as e:
        s.Setup(gpu.MAT(P.poisson2d(15)))
    assert e.value.code == -31


def test_two_grid_cycle_against_textbook_numpy(gpu):
    """An independent pin for MG with transfer operators: the two-grid cycle on 2D Poisson
    31 x 31 (bilinear P, R = P^T, A_c = R A P, weighted Jacobi 2/3 with 2 + 2 sweeps, 400
    Jacobi sweeps from zero on the 15 x 15 coarse grid, enough to make the coarse solve
    exact to ~1e-7) written here from the textbook algorithm
    with SciPy sparse products -- not from the reference or the oracle. The GPU, given only
    P, forms R and A_c itself. Bars: after one cycle x within 1e-12 of max|x|; the residual
    norms of 8 cycles within 1e-9 relative; the contraction per cycle below 0.2."""
    import scipy.sparse as sp
    nf, nc = 31, 15
    A = P.poisson2d(nf)
    S = A.scipy()
    rows, cols, vals = [], [], []
    for i in range(nf):  # 1D linear interpolation, coarse point j at fine point 2j + 1
        if i % 2 == 1:
            rows.append(i), cols.append((i - 1) // 2), vals.append(1.0)
        else:
            for j in (i // 2 - 1, i // 2):
                if 0 <= j < nc:
                    rows.append(i), cols.append(j), vals.append(0.5)
    p1 = sp.csr_matrix((vals, (rows, cols)), shape=(nf, nc))
    Pm = sp.kron(p1, p1, format="csr")  # x fastest: the second factor runs over x
    Pm.sort_indices()
    R = Pm.T.tocsr()
    Ac = (R @ S @ Pm).tocsr()

    def jacobi(M, b, x, sweeps):
        d = M.diagonal()
        for _ in range(sweeps):
            x = x + (2.0 / 3.0) * (b - M @ x) / d
        return x

    def cycle(x, b):
        x = jacobi(S, b, x, 2)
        ec = jacobi(Ac, R @ (b - S @ x), np.zeros(nc * nc), 400)
        return jacobi(S, b, x + Pm @ ec, 2)

    b = A.matvec(np.random.default_rng(11).uniform(-1, 1, A.nrow))
    gP = gpu.MAT(P.CSRMatrix(nf * nf, nc * nc, Pm.indptr.astype(np.uint32),
                             Pm.indices.astype(np.uint32), Pm.data.astype(np.float64)))
    M = gpu.MAT(A)
    kw = dict(KW, mgLevels=1, relTol=1e-300,
              mgCoarse=dict(maxIter=400, minIter=400, weight=2.0 / 3.0))
    for ncyc in (1, 8):
        s = gpu.configure("mg", **{**kw, "maxIter": ncyc})
        s.SetTransfer(0, gP, None, None)
        s.Setup(M)
        x = np.zeros(A.nrow)
        s.Solve(b, x)
        xn = np.zeros(A.nrow)
        res = [np.linalg.norm(b)]
        for _ in range(ncyc):
            xn = cycle(xn, b)
            res.append(np.linalg.norm(b - S @ xn))
        if ncyc == 1:
            assert np.max(np.abs(x - xn)) <= 1e-12 * np.max(np.abs(xn))
        else:
            h = s.History()[: ncyc + 1]
            assert np.allclose(h, res, rtol=1e-9, atol=0.0), (h, res)
            rates = np.array(res[1:]) / np.array(res[:-1])
            assert np.max(rates) < 0.2, rates
