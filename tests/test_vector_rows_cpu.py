"""Index arithmetic of the vector-row stencil kernels, checked on the CPU.

The kernels (cg_spmv's four-row FP32 and two-row FP64 paths, k_stencil_vec, bi_p / bi_s)
give each thread W consecutive rows (one 16-byte group), let the lanes of a warp hold
consecutive groups, take the -1/+1 neighbours from the adjacent lanes' groups by shuffles
(lanes 0 and 31 load the group beyond the warp), load the other offsets as aligned groups
(or two groups and a shift) with 32-bit wrapped indices bounded by one unsigned compare, and
-- for 7-point stencils whose plane stride is a multiple of 32 W -- walk columns of planes
(MarchPlan: chunk = ceil(planes x cols / threads)). This file restates that arithmetic in
Python and checks, for several matrices and grid sizes, that every group is processed
exactly once, that every load stays inside the vector, and that every row sees the right
value at every offset its mask holds. No GPU is involved.
"""
import numpy as np
import pytest

from faspxx_b200 import problems as P

M32 = 0xFFFFFFFF


def _offsets_masks(A):
    rows = np.repeat(np.arange(A.nrow, dtype=np.int64), np.diff(A.rowPtr.astype(np.int64)))
    d = A.colInd.astype(np.int64) - rows
    offs = sorted(set(d.tolist()))
    k = np.searchsorted(offs, d)
    mask = np.zeros(A.nrow, np.uint32)
    np.bitwise_or.at(mask, rows, (1 << k).astype(np.uint32))
    return offs, mask


def _shape(offs):
    """stencil_shape: 5 or 7 for [-S1, -1, 0, 1, S1] / [-S2, -S1, -1, 0, 1, S1, S2] with the
    S multiples of 4, else 0."""
    if len(offs) not in (5, 7):
        return 0
    mid = len(offs) // 2
    if offs[mid] != 0 or offs[mid - 1] != -1 or offs[mid + 1] != 1:
        return 0
    return len(offs) if all(o % 4 == 0 for k, o in enumerate(offs)
                            if k < mid - 1 or k > mid + 1) else 0


def _march_plan(offs, n, threads, rpg):
    if len(offs) != 7 or offs[0] != -offs[6]:
        return None
    s2 = offs[6]
    if s2 % (32 * rpg) or n % s2 or n // s2 < 2:
        return None
    cols, nz = s2 // rpg, n // s2
    return cols, nz, max(1, -(-(nz * cols) // threads))


def _check(A, W, threads, walk=True):
    """Runs the kernels' gather plan for rows grouped by W over `threads` threads; returns
    whether the plane walk was taken."""
    n = A.nrow
    assert n % W == 0
    offs, mask = _offsets_masks(A)
    nw = n // W
    vals = np.random.default_rng(0).standard_normal(n)
    grp = vals.reshape(nw, W)
    seen = np.zeros(nw, np.int64)

    def ld(h):
        assert 0 <= h < nw, h
        return grp[h]

    def verify(g, xs):
        seen[g] += 1
        for j in range(W):
            row = W * g + j
            for k, d in enumerate(offs):
                if (mask[row] >> k) & 1:
                    assert xs[k][j] == vals[row + d], (g, j, d)

    def neighbour_words(G, cur, l, act):
        g = G[l]
        last = cur[l - 1][W - 1] if l > 0 else (ld(g - 1)[W - 1] if act and g > 0 else 0.0)
        first = cur[l + 1][0] if l < 31 else (ld(g + 1)[0] if act and g + 1 < nw else 0.0)
        return last, first

    def gather(g, act, d, cur_l, last, first):
        if d == 0:
            return cur_l
        if d == -1:
            return np.concatenate([[last], cur_l[:W - 1]])
        if d == 1:
            return np.concatenate([cur_l[1:], [first]])
        q, s = d // W, d % W               # floor division, as d >> log2(W)
        ga = (g + q) & M32
        a = ld(ga) if act and ga < nw else np.zeros(W)
        if s == 0:
            return a
        gb = (ga + 1) & M32
        b = ld(gb) if act and gb < nw else np.zeros(W)
        return np.concatenate([a, b])[s:s + W]

    plan = _march_plan(offs, n, threads, W) if walk else None
    if plan:
        cols, nz, C = plan
        items = cols * -(-nz // C)
        assert items % 32 == 0
        for w0 in range(0, threads, 32):
            for w in range(w0, items, threads):          # whole warps
                k0 = (w // cols) * C
                k1 = min(k0 + C, nz)
                G = [(w + l) % cols + k0 * cols for l in range(32)]
                assert all(G[l] == G[0] + l for l in range(32))  # one plane, consecutive
                assert len({(w + l) // cols for l in range(32)}) == 1
                for _ in range(k0, k1):
                    cur = [ld(g) for g in G]
                    for l, g in enumerate(G):
                        last, first = neighbour_words(G, cur, l, True)
                        verify(g, [gather(g, True, d, cur[l], last, first) for d in offs])
                    G = [g + cols for g in G]
    else:
        for w0 in range(0, threads, 32):
            for g0 in range(w0, nw, threads):           # g - lane < nw: whole warps
                G = [g0 + l for l in range(32)]
                act = [g < nw for g in G]
                cur = [ld(g) if a else np.zeros(W) for g, a in zip(G, act)]
                for l, g in enumerate(G):
                    if not act[l]:
                        continue
                    last, first = neighbour_words(G, cur, l, True)
                    verify(g, [gather(g, True, d, cur[l], last, first) for d in offs])
    assert (seen == 1).all()
    return plan is not None


def _banded(n, offs):
    import scipy.sparse as sp
    B = sp.diags([np.full(n - abs(d), 1.0) for d in offs], offs, shape=(n, n), format="csr")
    B.sort_indices()
    return P.CSRMatrix(n, n, B.indptr.astype(np.uint32), B.indices.astype(np.uint32),
                       B.data.astype(np.float64))


@pytest.mark.parametrize("W", [4, 2])
@pytest.mark.parametrize("name,threads,walks", [
    ("poisson3d_16", 3 * 64, True),      # plane stride 256: walked for W = 4 and 2
    ("poisson3d_8", 2 * 64, None),       # plane stride 64: walked for W = 2 only
    ("poisson3d_12", 64, False),         # plane stride 144: not a multiple of 128 / 64
    ("poisson2d_40", 128, False),        # 5-point
])
def test_fixed_shapes_cover_every_group_once(W, name, threads, walks):
    A = {"poisson3d_16": P.poisson3d(16), "poisson3d_8": P.poisson3d(8),
         "poisson3d_12": P.poisson3d(12), "poisson2d_40": P.poisson2d(40)}[name]
    offs, _ = _offsets_masks(A)
    assert _shape(offs) in (5, 7)
    walked = _check(A, W, threads)
    if walks is None:
        assert walked == (W == 2)
    else:
        assert walked == walks
    if walked:
        assert not _check(A, W, threads, walk=False)  # the unwalked loop is right too


@pytest.mark.parametrize("offs,n", [
    ([-3, -2, -1, 0, 1, 2, 3], 400),      # shuffles reaching three elements each way
    ([-7, -2, 0, 3, 5], 300),             # unaligned offsets: two groups and a shift
    ([-1500, -7, -2, 0, 2, 7, 1500], 2048),
])
def test_generic_offsets_four_rows(offs, n):
    """The four-row FP32 kernel with generic offsets (no fixed shape). For |d| = 2, 3 the
    kernel shuffles the neighbouring lanes' words; the two-group form restated here reads
    the same elements (and bounds the loads the lanes at the warp's ends make)."""
    A = _banded(n, offs)
    assert _shape(_offsets_masks(A)[0]) == 0
    _check(A, 4, 64, walk=False)


def test_shape_and_plan_conditions():
    assert _shape([-256, -16, -1, 0, 1, 16, 256]) == 7
    assert _shape([-40, -1, 0, 1, 40]) == 5
    assert _shape([-100, -10, -1, 0, 1, 10, 100]) == 0   # 10 is not a multiple of 4
    assert _shape([-2, -1, 0, 1, 2]) == 0
    # 128^3: 4,096 four-row groups a plane, 128 planes over 444 blocks of 256 threads
    cols, nz, chunk = _march_plan([-16384, -128, -1, 0, 1, 128, 16384], 128 ** 3, 444 * 256, 4)
    assert (cols, nz, chunk) == (4096, 128, 5)
    assert cols * -(-nz // chunk) <= 444 * 256
    assert _march_plan([-9216, -96, -1, 0, 1, 96, 9216], 96 ** 3, 444 * 256, 4) is not None
    assert _march_plan([-10000, -100, -1, 0, 1, 100, 10000], 100 ** 3, 444 * 256, 4) is None
