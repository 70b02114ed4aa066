"""Block tiles of the CSR form: 256 rows per block, their row pointers, column indices and
values brought into shared memory by bulk asynchronous copies two tiles ahead of the
threads that sum the rows (faspxx_b200/csrc/common.cuh, csr_tile_rows).

Bar: bit-exact against the row-at-a-time kernels. Each row is still summed by one thread in
CSR order with one FMA per entry, and thread t still owns rows t, t + S, t + 2S, ... in that
order, so MAT::Apply, MAT::Residual and whole GMRES/FGMRES solves (whose Arnoldi products
take the tiles) give the same bits whether the tiles run or not. The row-at-a-time kernels are reached on the same matrix by switching on
the 16-bit column offsets (their kernels walk rows one at a time; the offsets change the
loads, not the arithmetic).
"""
import numpy as np
import pytest

from faspxx_b200 import problems as P

pytestmark = pytest.mark.gpu

CSR = 0


@pytest.fixture(scope="module")
def gpu():
    from faspxx_b200 import capi, sol
    capi.init(0)
    return sol


def _ragged(n, seed, maxlen=7, empty=0.05):
    """n rows of 0 to maxlen entries (a share of them empty) within 2,000 columns of the
    diagonal, values of both signs; square, so that Residual applies. Entry k of a row lies
    in the k-th window of 571 columns from row - 2000 (sorted, distinct); entries that fall
    outside the matrix are dropped."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, maxlen + 1, n)
    lens[rng.random(n) < empty] = 0
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    first = np.repeat(np.cumsum(lens) - lens, lens)
    k = np.arange(rows.size) - first
    cols = rows - 2000 + k * 571 + rng.integers(0, 571, rows.size)
    keep = (cols >= 0) & (cols < n)
    rows, cols = rows[keep], cols[keep]
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum(np.bincount(rows, minlength=n))
    va = rng.uniform(-1, 1, cols.size)
    return P.CSRMatrix(n, n, rp, cols.astype(np.uint32), va)


def _apply_both(gpu, A, seed=1):
    M = gpu.MAT(A)
    M.SetRowClass(CSR)
    rng = np.random.default_rng(seed)
    x = gpu.DVec.from_numpy(rng.standard_normal(A.mcol))
    b = gpu.DVec.from_numpy(rng.standard_normal(A.nrow))
    out = []
    for col16 in (False, True):
        M.SetCol16(col16)
        y, r = gpu.DVec(A.nrow), gpu.DVec(A.nrow)
        M.Apply(x, y)
        M.Residual(b, x, r)
        out.append((y.numpy(), r.numpy()))
    return M, x, out


@pytest.mark.parametrize("name,A", [
    ("poisson3d_20", P.poisson3d(20)),          # 8,000 rows: 32 tiles, the last one whole
    ("poisson3d_33", P.poisson3d(33)),          # 35,937 rows: a ragged last tile
    ("poisson2d_300", P.poisson2d(300)),        # 5-point rows
    ("ragged_70001", _ragged(70001, 3)),        # empty rows, lengths 0..7
])
def test_apply_residual_bit_exact(gpu, name, A):
    M, x, out = _apply_both(gpu, A)
    M.SetCol16(False)
    span, f64, f32, used = M.TileInfo()
    assert f64 and f32 and used and span <= 1812
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    ref = A.matvec(x.numpy())
    assert np.max(np.abs(out[0][0] - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))
    assert gpu.tile_timeouts() == 0


def test_tile_span_and_fallback(gpu):
    """A 2D 9-point stencil covers 2,304 entries per tile: no stage holds it, so the kernels
    walk rows one at a time; the result is still right."""
    A = P._from_stencil((120, 120, 1), [(dx, dy, 0) for dy in (-1, 0, 1) for dx in (-1, 0, 1)],
                        lambda k: 8.0 if k == 4 else -1.0)
    M = gpu.MAT(A)
    M.SetRowClass(CSR)
    span, f64, f32, used = M.TileInfo()
    assert span > 2000 and not f64 and not f32 and used
    x = np.random.default_rng(2).standard_normal(A.mcol)
    y = gpu.DVec(A.nrow)
    M.Apply(gpu.DVec.from_numpy(x), y)
    ref = A.matvec(x)
    assert np.max(np.abs(y.numpy() - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_many_tiles_per_block(gpu):
    """600,001 rows: more tiles than blocks, so every block runs its two stages round and
    round (both mbarrier phases, stage reuse after the block barrier)."""
    A = _ragged(600_001, 8, maxlen=6)
    _, _, out = _apply_both(gpu, A, seed=4)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    assert gpu.tile_timeouts() == 0


@pytest.mark.parametrize("alg,prec", [("gmres", "FP64"), ("gmres", "MIXED"),
                                      ("fgmres", "FP64")])
def test_gmres_solve_bit_exact(gpu, alg, prec):
    """GMRES(30) and FGMRES on the CSR form of a 64^3 convection-diffusion matrix (1,024
    tiles: more than one per block): the Arnoldi products take the tiles; iterations,
    solution and history must equal those of the same solve with the tiles off."""
    from faspxx_b200 import capi
    A = P.convdiff3d(64, 1.0)
    b = A.matvec(np.random.default_rng(6).uniform(-1, 1, A.nrow))
    out = []
    for col16 in (False, True):
        M = gpu.MAT(A)
        M.SetRowClass(CSR)
        M.SetCol16(col16)
        s = gpu.configure(alg, maxIter=600, relTol=1e-8, absTol=0.0, restart=30,
                          pcd="jacobi", pcdWeight=2.0 / 3.0, pcdIter=1)
        s.SetPrecision(getattr(capi, prec))
        s.Setup(M)
        x = np.zeros(A.nrow)
        code = s.Solve(b, x)
        out.append((code, s.GetIterations(), x, np.nan_to_num(s.History())))
        if not col16:
            assert M.TileInfo()[3]
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][3], out[1][3])
    assert gpu.tile_timeouts() == 0
