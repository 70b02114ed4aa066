"""The DCGS2 Arnoldi recurrences (classical Gram-Schmidt with the reorthogonalisation delayed
into the next step), restated in numpy exactly as the GPU passes form them (dcgs2.cu), held
against the reference's modified Gram-Schmidt Arnoldi (GMRES.cxx:160-210) on the same
operator: the Givens residual estimates of a 30-step cycle agree to 1e-8 relative (above a
floor of rounding in ||r0||), the basis is orthonormal to rounding, and a lucky breakdown
(t = 0) ends with the estimate at rounding level instead of NaN. Step j: a = Q^T u,
b = Q^T w, c = u^T w, d = u^T u; t = sqrt(d - a^T a); column j - 1 += a with subdiagonal t;
h = (b - H a) / t,
h_j = ((c - a^T b) / t - t a_{j-1}) / t; q_j = (u - Q a) / t; u_{j+1} = (w - Q b - q_j g) / t
with g = (c - a^T b) / t.
"""
import numpy as np
import scipy.sparse as sp


def _givens(col, count, c1, hc, hs, var):
    """The reference's Givens step on Hessenberg column c1 (GMRES.cxx:168-203)."""
    for j in range(1, count):
        t = col[j - 1]
        col[j - 1] = hs[j - 1] * col[j] + hc[j - 1] * t
        col[j] = -hs[j - 1] * t + hc[j - 1] * col[j]
    t = np.sqrt(col[count] ** 2 + col[c1] ** 2)
    hc[c1], hs[c1] = col[c1] / t, col[count] / t
    col[c1] = hs[c1] * col[count] + hc[c1] * col[c1]
    var[count] = -hs[c1] * var[c1]
    var[c1] = hc[c1] * var[c1]
    return abs(var[count])


def _cycle_mgs(A, r0, m):
    n = A.shape[0]
    beta = np.linalg.norm(r0)
    V = np.zeros((m + 1, n))
    V[0] = r0 / beta
    H = np.zeros((m + 1, m))
    hc, hs, var = np.zeros(m + 1), np.zeros(m), np.zeros(m + 1)
    var[0] = beta
    est = []
    for j in range(m):
        w = A @ V[j]
        for i in range(j + 1):
            H[i, j] = V[i] @ w
            w = w - H[i, j] * V[i]
        H[j + 1, j] = np.linalg.norm(w)
        V[j + 1] = w / H[j + 1, j]
        est.append(_givens(H[:, j].copy(), j + 1, j, hc, hs, var))
    return np.array(est), V[:m]


def _cycle_dcgs2(A, r0, m):
    n = A.shape[0]
    beta = np.linalg.norm(r0)
    V = np.zeros((m + 1, n))
    V[0] = r0 / beta
    Hraw = np.zeros((m + 1, m))
    hc, hs, var = np.zeros(m + 1), np.zeros(m), np.zeros(m + 1)
    var[0] = beta
    est = []
    for j in range(m + 1):
        has_w = j < m
        u, Q = V[j].copy(), V[:j]
        w = A @ u if has_w else None
        a, d = Q @ u, u @ u
        if j >= 1:
            t = np.sqrt(max(d - a @ a, 0.0))
            Hraw[:j, j - 1] += a
            Hraw[j, j - 1] = t
            est.append(_givens(Hraw[:, j - 1].copy(), j, j - 1, hc, hs, var))
            tinv = 1.0 / t if t > 0 else np.inf
        else:
            t, tinv = 1.0, 1.0
        if not has_w or (j >= 1 and est[-1] == 0.0):
            break
        b, c = Q @ w, u @ w
        if j >= 1:
            h = np.zeros(j + 1)
            h[:j] = (b - Hraw[:j, :j] @ a) * tinv
            g = (c - a @ b) * tinv
            h[j] = (g - t * a[j - 1]) * tinv
            q = (u - Q.T @ a) * tinv
            un = (w - Q.T @ b - q * g) * tinv
        else:
            h, g, q, un = np.array([c]), c, u, w - u * c
        Hraw[: j + 1, j] = h
        V[j], V[j + 1] = q, un
    return np.array(est), V[:m]


def _convdiff(n, seed):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=0.02, random_state=seed) + sp.eye(n) * 4.0
    return A.tocsr(), rng.standard_normal(n)


def test_dcgs2_estimates_match_mgs():
    A, b = _convdiff(400, 3)
    e_mgs, _ = _cycle_mgs(A, b, 30)
    e_dc, V = _cycle_dcgs2(A, b, 30)
    assert len(e_dc) == 30
    # relative agreement, down to a floor of rounding in ||r0|| (the last estimates are
    # about 1e-12 of it and carry the rounding of 30 steps, as CGS2's do)
    beta = np.linalg.norm(b)
    assert np.all(np.abs(e_dc - e_mgs) <= 1e-8 * np.abs(e_mgs) + 1e-16 * beta)
    assert np.linalg.norm(V @ V.T - np.eye(30)) < 1e-13


def test_dcgs2_lucky_breakdown():
    """Three distinct eigenvalues: the Krylov space is exhausted after three steps and the
    estimate falls to rounding (no NaN reaches it)."""
    d = np.concatenate([np.full(100, 1.0), np.full(150, 2.0), np.full(150, 5.0)])
    A = sp.diags(d).tocsr()
    b = np.random.default_rng(1).standard_normal(400)
    with np.errstate(all="ignore"):
        e_dc, _ = _cycle_dcgs2(A, b, 6)
    assert np.all(np.isfinite(e_dc))
    assert e_dc[2] < 1e-13 * np.linalg.norm(b)
