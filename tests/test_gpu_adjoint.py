"""Differentiable solve: adjoint CG on the exact transpose + sampled outer product, checked
against central finite differences and an FP64 reference gradient (SciPy sparse direct
solves on the CPU). Workload: variable-coefficient diffusion -div(kappa grad u) = b on an
N^3 grid, kappa = exp(N(0,1)) per cell, harmonic face averages; loss 1/2 ||x - x_t||^2.

Tolerances: gradient vs the FP64 reference <= 1e-6 relative (forward/adjoint CG to
rtol 1e-12); directional derivative vs central differences (eps = 1e-6 relative step)
<= 1e-5 relative, 32 seeded directions.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    from faspxx_b200 import autograd as AG
    from faspxx_b200 import problems as P
    N = 12
    rng = np.random.default_rng(0)
    kappa = np.exp(rng.standard_normal(N ** 3))
    A = P.vardiff3d(N, kappa)
    b = rng.standard_normal(A.nrow)
    xt = rng.standard_normal(A.nrow)
    sysm = AG.SparseSystem(A.rowPtr, A.colInd, A.nrow, relTol=1e-12)
    return torch, AG, P, A, b, xt, sysm


def loss_of(torch, AG, sysm, vals, b, xt):
    x = AG.sparse_solve(vals, b, sysm)
    return 0.5 * torch.sum((x - xt) ** 2), x


def test_gradient_matches_fp64_reference(setup):
    torch, AG, P, A, b, xt, sysm = setup
    import scipy.sparse.linalg as spla
    dev = "cuda:0"
    vals = torch.tensor(A.values, device=dev, requires_grad=True)
    bt = torch.tensor(b, device=dev, requires_grad=True)
    xtt = torch.tensor(xt, device=dev)
    L, x = loss_of(torch, AG, sysm, vals, bt, xtt)
    L.backward()
    S = A.scipy().tocsc()
    xr = spla.spsolve(S, b)
    lam = spla.spsolve(S.T.tocsc(), xr - xt)
    rows = np.repeat(np.arange(A.nrow), np.diff(A.rowPtr.astype(np.int64)))
    dA = -lam[rows] * xr[A.colInd]
    gA = vals.grad.cpu().numpy()
    gb = bt.grad.cpu().numpy()
    assert np.linalg.norm(x.detach().cpu().numpy() - xr) <= 1e-9 * np.linalg.norm(xr)
    assert np.linalg.norm(gb - lam) <= 1e-6 * np.linalg.norm(lam)
    assert np.linalg.norm(gA - dA) <= 1e-6 * np.linalg.norm(dA)


def test_central_differences_32_directions(setup):
    torch, AG, P, A, b, xt, sysm = setup
    dev = "cuda:0"
    vals = torch.tensor(A.values, device=dev, requires_grad=True)
    bt = torch.tensor(b, device=dev, requires_grad=True)
    xtt = torch.tensor(xt, device=dev)
    L, _ = loss_of(torch, AG, sysm, vals, bt, xtt)
    L.backward()
    gA, gb = vals.grad.clone(), bt.grad.clone()
    rng = np.random.default_rng(1)
    worst = 0.0
    for _ in range(32):
        # symmetric perturbation of the matrix keeps it SPD for CG
        dv = rng.standard_normal(A.nnz) * np.abs(A.values)
        S = A.scipy()
        D = type(S)((dv, A.colInd, A.rowPtr), shape=S.shape)
        D = (D + D.T) * 0.5
        D = D.tocsr()
        D.sort_indices()
        dvs = torch.tensor(np.asarray(D[A.scipy().nonzero()]).ravel() if False else
                           _on_pattern(A, D), device=dev)
        db = torch.tensor(rng.standard_normal(A.nrow), device=dev)
        eps = 1e-6
        with torch.no_grad():
            Lp, _ = loss_of(torch, AG, sysm, vals + eps * dvs, bt + eps * db, xtt)
            Lm, _ = loss_of(torch, AG, sysm, vals - eps * dvs, bt - eps * db, xtt)
        fd = (Lp - Lm).item() / (2 * eps)
        an = (torch.dot(gA, dvs) + torch.dot(gb, db)).item()
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-30))
    assert worst <= 1e-5, worst


def _on_pattern(A, D):
    """Values of sparse matrix D at A's stored positions (A's pattern contains D's)."""
    rows = np.repeat(np.arange(A.nrow), np.diff(A.rowPtr.astype(np.int64)))
    return np.asarray(D[rows, A.colInd.astype(np.int64)]).ravel()


def test_adjoint_uses_transpose_of_nonsymmetric(setup):
    """On a nonsymmetric matrix the adjoint must solve with A^T, not A."""
    torch, AG, P, A, b, xt, sysm = setup
    import scipy.sparse.linalg as spla
    from faspxx_b200 import capi, sol
    C = P.convdiff3d(8, 2.0)
    M = sol.MAT(C)
    s = sol.configure("gmres", maxIter=2000, relTol=1e-12, absTol=0.0, restart=30,
                      maxRestart=30, minRestart=30, pcd="jacobi", pcdWeight=2 / 3)
    s.Setup(M)
    g = np.random.default_rng(3).standard_normal(C.nrow)
    lam = sol.DVec(C.nrow)
    code = s.SolveAdjoint(sol.DVec.from_numpy(g), lam)
    assert code == 0
    ref = spla.spsolve(C.scipy().T.tocsc(), g)
    assert np.linalg.norm(lam.numpy() - ref) <= 1e-9 * np.linalg.norm(ref)
