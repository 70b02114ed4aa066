"""Host-side CSRx containers and the synthetic sparse problems used by tests and bench.

``CSRMatrix`` holds a CSRx matrix the way FASP++'s MAT does (src/MAT.hxx:43-47): 32-bit
unsigned row pointers and column indices, columns ascending in every row and the diagonal
always stored. The generators build the five workloads of the iterative-solve path with
seeded NumPy random numbers; there is no external dataset.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class CSRMatrix:
    nrow: int
    mcol: int
    rowPtr: np.ndarray          # uint32[nrow+1]
    colInd: np.ndarray          # uint32[nnz]
    values: np.ndarray | None   # float64[nnz]; None = pattern only

    @property
    def nnz(self) -> int:
        return int(self.colInd.shape[0])

    def scipy(self):
        import scipy.sparse as sp
        vals = self.values if self.values is not None else np.ones(self.nnz)
        return sp.csr_matrix((vals, self.colInd.astype(np.int64), self.rowPtr.astype(np.int64)),
                             shape=(self.nrow, self.mcol))

    def matvec(self, x):
        return self.scipy() @ np.asarray(x, dtype=np.float64)

    def diag_ptr(self) -> np.ndarray:
        """Position of the diagonal in each row (MAT::FormDiagPtr, src/MAT.cxx:917-928)."""
        rows = np.repeat(np.arange(self.nrow, dtype=np.int64), np.diff(self.rowPtr.astype(np.int64)))
        hit = np.nonzero(self.colInd.astype(np.int64) == rows)[0]
        dp = np.zeros(self.nrow, dtype=np.uint32)
        # the first match in each row wins, like the linear search
        r = rows[hit]
        first = np.ones(len(hit), dtype=bool)
        first[1:] = r[1:] != r[:-1]
        dp[r[first]] = hit[first]
        return dp


def _from_stencil(shape, offsets, coef):
    """CSR of a structured-grid stencil in lexicographic order (x fastest).

    offsets: list of (dx, dy, dz) in ascending column order; coef(k) -> array[n] of the
    values of neighbour k (entries whose neighbour is outside the grid are dropped).
    """
    nx, ny, nz = shape
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64)
    ix, iy, iz = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    cols, vals, valid = [], [], []
    for k, (dx, dy, dz) in enumerate(offsets):
        ok = (ix + dx >= 0) & (ix + dx < nx) & (iy + dy >= 0) & (iy + dy < ny) & \
             (iz + dz >= 0) & (iz + dz < nz)
        cols.append(idx + dx + dy * nx + dz * nx * ny)
        vals.append(np.broadcast_to(coef(k), (n,)))
        valid.append(ok)
    cols = np.stack(cols, axis=1)
    vals = np.stack(vals, axis=1)
    valid = np.stack(valid, axis=1)
    counts = valid.sum(axis=1)
    rowPtr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowPtr[1:])
    colInd = cols[valid].astype(np.uint32)
    values = np.ascontiguousarray(vals[valid], dtype=np.float64)
    return CSRMatrix(n, n, rowPtr.astype(np.uint32), colInd, values)


_OFF2D = [(0, -1, 0), (-1, 0, 0), (0, 0, 0), (1, 0, 0), (0, 1, 0)]
_OFF3D = [(0, 0, -1), (0, -1, 0), (-1, 0, 0), (0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]


def poisson2d(nx: int, ny: int | None = None, shift: float = 0.0) -> CSRMatrix:
    """5-point FDM Laplacian, diagonal 4 (+shift), off-diagonals -1, Dirichlet boundary."""
    ny = nx if ny is None else ny
    c = [-1.0, -1.0, 4.0 + shift, -1.0, -1.0]
    return _from_stencil((nx, ny, 1), _OFF2D, lambda k: c[k])


def poisson3d(nx: int, ny: int | None = None, nz: int | None = None) -> CSRMatrix:
    """7-point FDM Laplacian, diagonal 6, off-diagonals -1, Dirichlet boundary."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    c = [-1.0, -1.0, -1.0, 6.0, -1.0, -1.0, -1.0]
    return _from_stencil((nx, ny, nz), _OFF3D, lambda k: c[k])


def convdiff3d(N: int, peclet: float, direction=(1.0, 0.5, 0.25)) -> CSRMatrix:
    """-Laplace(u) + beta.grad(u) on an N^3 interior grid, h = 1/(N+1), first-order upwind.

    beta = s * direction with s chosen so that the cell Peclet number
    |beta|_inf * h / 2 equals ``peclet``. Rows are scaled like the operator (1/h^2 and 1/h).
    """
    h = 1.0 / (N + 1)
    d = np.asarray(direction, dtype=np.float64)
    beta = d * (2.0 * peclet / h / np.abs(d).max())
    inv_h2, inv_h = 1.0 / (h * h), 1.0 / h
    # upwind: beta_i > 0 uses the backward difference (u_j - u_{j-1})/h
    c = np.zeros(7)
    c[3] = 6.0 * inv_h2
    for axis, (lo, hi) in enumerate(((2, 4), (1, 5), (0, 6))):
        c[lo] = -inv_h2
        c[hi] = -inv_h2
        b = beta[axis]
        if b >= 0:
            c[3] += b * inv_h
            c[lo] -= b * inv_h
        else:
            c[3] -= b * inv_h
            c[hi] += b * inv_h
    return _from_stencil((N, N, N), _OFF3D, lambda k: c[k])


def vardiff3d(N: int, kappa: np.ndarray) -> CSRMatrix:
    """-div(kappa grad u) on an N^3 cell grid, h = 1/(N+1), Dirichlet boundary.

    kappa holds one coefficient per cell; interior faces use the harmonic mean of the two
    cells, boundary faces the cell's own value. The matrix is SPD.
    """
    n = N ** 3
    h2 = 1.0 / (N + 1) ** 2
    k = np.asarray(kappa, dtype=np.float64).reshape(n)
    idx = np.arange(n, dtype=np.int64)
    ix, iy, iz = idx % N, (idx // N) % N, idx // (N * N)
    diag = np.zeros(n)
    face = []
    for (dx, dy, dz) in _OFF3D:
        if (dx, dy, dz) == (0, 0, 0):
            face.append(None)
            continue
        ok = (ix + dx >= 0) & (ix + dx < N) & (iy + dy >= 0) & (iy + dy < N) & \
             (iz + dz >= 0) & (iz + dz < N)
        j = np.where(ok, idx + dx + dy * N + dz * N * N, idx)
        kf = np.where(ok, 2.0 * k * k[j] / (k + k[j]), k)
        diag += kf
        face.append(-kf)
    coefs = [diag / h2 if f is None else f / h2 for f in face]
    return _from_stencil((N, N, N), _OFF3D, lambda kk: coefs[kk])


def rhs_from_solution(A: CSRMatrix, xstar: np.ndarray) -> np.ndarray:
    return A.matvec(xstar)


def seeded_uniform(n: int, seed: int = 42, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    return np.random.default_rng(seed).uniform(lo, hi, n)


def batch_systems(count: int = 4096, mlo: int = 16, mhi: int = 128, nrhs: int = 4,
                  seed: int = 42):
    """The batched workload: ``count`` 2D 5-point Poisson systems on m x m grids, m ~ U{mlo..mhi},
    each shifted by sigma*I with sigma ~ U[0,1], with ``nrhs`` right-hand sides b ~ N(0,1).

    Returns (ms, sigmas, rhs) where rhs[i] has shape (nrhs, m_i^2).
    """
    rng = np.random.default_rng(seed)
    ms = rng.integers(mlo, mhi + 1, size=count)
    sig = rng.uniform(0.0, 1.0, size=count)
    rhs = [rng.standard_normal((nrhs, int(m) * int(m))) for m in ms]
    return ms, sig, rhs


def read_csr_raw(path: str):
    """The arrays ReadCSR (src/ReadData.cxx:221-358) reads from a text CSR file, before any
    conversion: n, then rowPtr[n + 1], colInd[nnz], values[nnz] as stored in the file
    (0- or 1-based, each row's entries in file order). Returns (n, rowPtr, colInd, values)."""
    with open(path) as f:
        tok = f.read().split()
    n = int(tok[0])
    rp = np.array(tok[1:n + 2], dtype=np.int64)
    nnz = int(rp[n] - rp[0])
    ci = np.array(tok[n + 2:n + 2 + nnz], dtype=np.int64)
    va = np.array(tok[n + 2 + nnz:n + 2 + 2 * nnz], dtype=np.float64)
    return n, rp.astype(np.uint32), ci.astype(np.uint32), va


def read_mtx_raw(path: str):
    """The triplets ReadMTX (src/ReadData.cxx:98-218) reads from a MatrixMarket file: lines
    starting with '%' skipped, then 'nrow mcol nnz', then nnz lines 'i j value' with 1-based
    indices, returned 0-based in file order: (nrow, mcol, rowInd, colInd, values)."""
    with open(path) as f:
        lines = [ln for ln in f if not ln.startswith("%")]
    tok = " ".join(lines).split()
    nrow, mcol, nnz = int(tok[0]), int(tok[1]), int(tok[2])
    t = np.array(tok[3:3 + 3 * nnz], dtype=object).reshape(nnz, 3)
    ri = t[:, 0].astype(np.int64) - 1
    ci = t[:, 1].astype(np.int64) - 1
    va = t[:, 2].astype(np.float64)
    return nrow, mcol, ri.astype(np.uint32), ci.astype(np.uint32), va


def read_csr_text(path: str) -> CSRMatrix:
    """FASP++ ReadMat of a text CSR file (src/ReadData.cxx:221-446): n, then n+1 row
    pointers, nnz column indices and nnz values; 1-based indices are shifted to 0-based,
    each row is sorted by column with a stable sort (SortCSRRow, src/MATUtil.cxx:439-476)
    and a zero diagonal is inserted where a row has none (CSRtoMAT, MATUtil.cxx:303-413)."""
    with open(path) as f:
        tok = f.read().split()
    n = int(tok[0])
    rp = np.array(tok[1:n + 2], dtype=np.int64)
    nnz = int(rp[n] - rp[0])
    ci = np.array(tok[n + 2:n + 2 + nnz], dtype=np.int64)
    va = np.array(tok[n + 2 + nnz:n + 2 + 2 * nnz], dtype=np.float64)
    if rp[0] == 1:
        rp -= 1
        ci -= 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    order = np.lexsort((ci, rows))          # by row, then column; stable
    ci, va = ci[order], va[order]
    has_diag = np.zeros(n, dtype=bool)
    has_diag[rows[ci == rows]] = True
    if not has_diag.all():
        missing = np.nonzero(~has_diag)[0]
        rows = np.concatenate([rows, missing])
        ci = np.concatenate([ci, missing])
        va = np.concatenate([va, np.zeros(len(missing))])
        order = np.lexsort((ci, rows))
        rows, ci, va = rows[order], ci[order], va[order]
        rp = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    return CSRMatrix(n, n, rp.astype(np.uint32), ci.astype(np.uint32), va)
