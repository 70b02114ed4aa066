"""Generate the golden fixtures under tests/golden/ from the FASP++ reference itself.

Run in a container that has the reference tree (given as the first argument or in
FASPXX_REFERENCE) after ``make -C oracle``; the GPU box never runs this script, it only
reads its outputs:

* ``fdm_10X10.npz``, ``fem_small.npz`` -- the reference's bundled matrices
  (data/fdm_10X10.csr, data/fem_small.csr) as 0-based uint32/float64 CSR arrays;
* ``known_answers.json`` -- the small known-answer cases of the reference's unit tests
  (utest/src/UnitTestsMAT.cxx:42-67,152-161; utest/src/UnitTestsJacobi.cxx:23-157;
  example/TestWeightedJacobi.cxx:60-136);
* ``reference_runs.npz`` + ``reference_runs.json`` -- outputs of the compiled reference
  (oracle/_ref/liboracle_ref.so) for every solver configuration the tests replay: return
  code, iteration count, norms, the solution x and the printed residual history;
* ``reference_transpose.npz`` -- MAT::TransInPlace results, the bit-exact target for CSC;
* ``reference_ingest.npz`` + ``reference_ingest.json`` -- ReadMat's conversions run by the
  reference (MTXtoMAT; ReadCSR's shift + SortCSRRow + CSRtoMAT) on the bundled data/*.csr
  and data/nos7.mtx arrays and on seeded synthetic inputs: shuffled entries, duplicates,
  missing and empty-row diagonals, long rows, rectangular and invalid matrices.

* ``reference_matfree.json`` -- what the reference's matrix-free example prints
  (example/TestMatFree.cxx, built from the reference sources by oracle/build_ref.sh).

* ``reference_mult.npz`` + ``reference_mult.json`` -- MAT::Mult products and MAT::Add sums
  computed by the reference (stencil squares, rectangular random factors, an interpolation
  product; stencil plus diagonal, unsorted random rows, repeated appended columns).

* ``reference_mta.npz`` + ``reference_mta.json`` -- MAT::MultTransposeAdd, v = A^T v1 + v2,
  computed by the reference on five structurally symmetric matrices and one that is not.

    python tests/golden/make_golden.py /path/to/reference
                                       [--runs-only | --ingest-only | --matfree-only |
                                        --mult-only]
    python tests/golden/make_golden.py --mta-only
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from faspxx_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden import cases as G  # noqa: E402


def check_against_readmat(path: str, A: P.CSRMatrix) -> None:
    """The Python reader must give exactly the MAT the reference's ReadMat builds."""
    lib = O.load("ref")
    nrow, nnz = C.c_uint32(), C.c_uint32()
    lib.orc_ref_readmat.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                    C.c_void_p, C.c_void_p, C.c_void_p]
    assert lib.orc_ref_readmat(path.encode(), C.byref(nrow), C.byref(nnz), None, None, None) == 0
    rp = np.empty(nrow.value + 1, np.uint32)
    ci = np.empty(nnz.value, np.uint32)
    va = np.empty(nnz.value, np.float64)
    lib.orc_ref_readmat(path.encode(), C.byref(nrow), C.byref(nnz), rp.ctypes.data,
                        ci.ctypes.data, va.ctypes.data)
    assert np.array_equal(rp, A.rowPtr) and np.array_equal(ci, A.colInd)
    assert np.array_equal(va, A.values)


def main(ref_root: str) -> None:
    O.build(ref=True)
    mats = {}
    for name in ("fdm_10X10", "fem_small"):
        path = os.path.join(ref_root, "data", name + ".csr")
        A = P.read_csr_text(path)
        check_against_readmat(path, A)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), rowPtr=A.rowPtr,
                            colInd=A.colInd, values=A.values)
        mats[name] = A

    runs_meta, runs_arr = {}, {}
    for case in G.solver_cases():
        A, b, x0 = G.case_inputs(case)
        s = O.Solver("ref", A, case["alg"], **case["kw"])
        outs = []
        for rep in range(case.get("repeat", 1)):
            r = s.solve(b, x0)
            outs.append(r)
        for rep, r in enumerate(outs):
            key = case["name"] if rep == 0 else f"{case['name']}__rep{rep}"
            runs_meta[key] = dict(code=r.code, iters=r.iters, norm2=r.norm2, normInf=r.normInf)
            runs_arr[key + "__x"] = r.x
            runs_arr[key + "__hist"] = r.hist
        if case.get("store_b"):
            runs_arr[case["name"] + "__b"] = b
    np.savez_compressed(os.path.join(HERE, "reference_runs.npz"), **runs_arr)
    with open(os.path.join(HERE, "reference_runs.json"), "w") as f:
        json.dump(runs_meta, f, indent=1, sort_keys=True)

    tr = {}
    for name, A in G.transpose_cases():
        rp, ci, va, dp = O.transpose("ref", A)
        tr[name + "__rowPtr"], tr[name + "__colInd"], tr[name + "__diagPtr"] = rp, ci, dp
        if va is not None:
            tr[name + "__values"] = va
    np.savez_compressed(os.path.join(HERE, "reference_transpose.npz"), **tr)
    print("wrote", len(runs_meta), "solver runs and", len(G.transpose_cases()), "transposes")


def _front_row0(ri, ci, order):
    """Reorders the entries so that row 0's first entry has its smallest column: the
    reference's SortCSRRow indexes out of bounds when an entry moves to the front of row 0."""
    order = list(order)
    pos = [k for k, j in enumerate(order) if ri[j] == 0]
    if pos:
        best = min(pos, key=lambda k: (ci[order[k]], k))
        order[pos[0]], order[best] = order[best], order[pos[0]]
    return np.array(order, dtype=np.int64)


def _coo(A: P.CSRMatrix):
    rows = np.repeat(np.arange(A.nrow, dtype=np.int64), np.diff(A.rowPtr.astype(np.int64)))
    return rows, A.colInd.astype(np.int64), A.values.copy()


def _random_coo(rng, nrow, mcol, per_row, dup=0.1, drop_diag=0.2, empty=0.05):
    """Random entries per row, some duplicated (same column, new value), some rows without
    their diagonal, some rows empty (never row 0)."""
    ri, ci = [], []
    for r in range(nrow):
        if r > 0 and rng.random() < empty:
            continue
        k = int(rng.integers(1, per_row + 1))
        cols = list(rng.choice(mcol, size=min(k, mcol), replace=False))
        if r < mcol:
            if rng.random() < drop_diag:
                cols = [c for c in cols if c != r] or [(r + 1) % mcol]
            elif r not in cols:
                cols.append(r)
        cols += [c for c in cols if rng.random() < dup]
        ri += [r] * len(cols)
        ci += cols
    ri, ci = np.array(ri, np.int64), np.array(ci, np.int64)
    va = rng.standard_normal(len(ri))
    return ri, ci, va


def ingest_cases(ref_root: str):
    """(name, kind, nrow, mcol, arrays) of every ingestion case; arrays are the reader's
    output: (rowInd, colInd, values) for "mtx", (rowPtr, colInd, values) for "csr"."""
    rng = np.random.default_rng(2024)
    out = []
    nr, mc, ri, ci, va = P.read_mtx_raw(os.path.join(ref_root, "data", "nos7.mtx"))
    out.append(("nos7_mtx", "mtx", nr, mc, (ri, ci, va)))
    for name in ("fdm_10X10", "fem_small"):
        n, rp, ci, va = P.read_csr_raw(os.path.join(ref_root, "data", name + ".csr"))
        out.append((name + "_csr", "csr", n, n, (rp, ci, va)))
    # a stencil matrix with its triplets in random order
    r, c, v = _coo(P.poisson2d(12))
    o = _front_row0(r, c, rng.permutation(len(r)))
    out.append(("poisson2d_shuffled_mtx", "mtx", 144, 144, (r[o], c[o], v[o])))
    # duplicates, missing diagonals, empty rows
    r, c, v = _random_coo(rng, 60, 60, 6)
    o = _front_row0(r, c, rng.permutation(len(r)))
    out.append(("random_dup_mtx", "mtx", 60, 60, (r[o], c[o], v[o])))
    # wide: every row can take its diagonal
    r, c, v = _random_coo(rng, 30, 47, 8)
    o = _front_row0(r, c, rng.permutation(len(r)))
    out.append(("wide_mtx", "mtx", 30, 47, (r[o], c[o], v[o])))
    # tall: rows >= mcol have no diagonal place, CSRtoMAT's check fails (MAT left empty)
    r, c, v = _random_coo(rng, 40, 30, 5)
    o = _front_row0(r, c, rng.permutation(len(r)))
    out.append(("tall_mtx", "mtx", 40, 30, (r[o], c[o], v[o])))
    # a column out of range: CheckCSR fails (MAT left empty)
    r, c, v = _random_coo(rng, 20, 20, 4)
    c = c.copy()
    c[len(c) // 2] = 20
    o = _front_row0(r, c, np.arange(len(r)))
    out.append(("badcol_mtx", "mtx", 20, 20, (r[o], c[o], v[o])))
    # long rows: 33..4096 (one block per row), > 4096 (merge passes), duplicates included
    lens = [3, 40, 700, 4096, 4097, 8300, 5, 1, 900]
    ri, ci = [], []
    for row, k in enumerate(lens):
        cols = rng.integers(0, 5000, size=k)
        if row == 0:
            cols[0] = cols.min()
        ri += [row] * k
        ci += list(cols)
    ri, ci = np.array(ri, np.int64), np.array(ci, np.int64)
    va = rng.integers(-64, 65, size=len(ri)) / 8.0  # short fixtures: few distinct values
    o = rng.permutation(len(ri))
    o = _front_row0(ri, ci, o)
    out.append(("long_rows_mtx", "mtx", len(lens), 5000, (ri[o], ci[o], va[o])))
    # raw CSR: rows shuffled in place, 0-based and 1-based, missing diagonals, duplicates
    for base, name in ((0, "shuffled0_csr"), (1, "dup1_csr")):
        if base == 0:
            A = P.poisson3d(5)
            r, c, v = _coo(A)
        else:
            r, c, v = _random_coo(rng, 50, 50, 7)
            o = np.lexsort((rng.random(len(r)), r))
            r, c, v = r[o], c[o], v[o]
        n = int(r.max()) + 1 if base == 0 else 50
        rp = np.zeros(n + 1, np.int64)
        np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
        c, v = c.copy(), v.copy()
        for i in range(n):
            seg = np.arange(rp[i], rp[i + 1])
            perm = rng.permutation(seg)
            if i == 0 and len(perm):
                k = int(np.argmin(c[perm]))
                perm[0], perm[k] = perm[k], perm[0]
            c[seg], v[seg] = c[perm], v[perm]
        out.append((name, "csr", n, n, (rp + base, c + base, v)))
    return out


def make_ingest(ref_root: str) -> None:
    O.build(ref=True)
    meta, arr = {}, {}
    for name, kind, nrow, mcol, (a, b, v) in ingest_cases(ref_root):
        if kind == "mtx":
            code, res = O.mtx_to_mat("ref", nrow, mcol, a, b, v)
        else:
            code, res = O.csr_to_mat("ref", nrow, a, b, v)
        assert code != O.REF_UNDEFINED, name
        meta[name] = dict(kind=kind, nrow=int(nrow), mcol=int(mcol), code=int(code),
                          nnz=0 if res is None else int(len(res[1])))
        arr[name + "__in0"] = np.asarray(a, np.uint32)
        arr[name + "__in1"] = np.asarray(b, np.uint32)
        arr[name + "__in2"] = np.asarray(v, np.float64)
        if res is not None:
            arr[name + "__rowPtr"], arr[name + "__colInd"], arr[name + "__values"] = res
    # the file reader itself on the bundled MatrixMarket file (ReadMat end to end)
    A = P.read_mtx_raw(os.path.join(ref_root, "data", "nos7.mtx"))
    code, res = O.mtx_to_mat("ref", *A)
    lib = O.load("ref")
    nrow, nnz = C.c_uint32(), C.c_uint32()
    lib.orc_ref_readmat.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                    C.c_void_p, C.c_void_p, C.c_void_p]
    path = os.path.join(ref_root, "data", "nos7.mtx").encode()
    assert lib.orc_ref_readmat(path, C.byref(nrow), C.byref(nnz), None, None, None) == 0
    rp = np.empty(nrow.value + 1, np.uint32)
    ci = np.empty(nnz.value, np.uint32)
    va = np.empty(nnz.value, np.float64)
    lib.orc_ref_readmat(path, C.byref(nrow), C.byref(nnz), rp.ctypes.data, ci.ctypes.data,
                        va.ctypes.data)
    assert np.array_equal(rp, res[0]) and np.array_equal(ci, res[1]) and np.array_equal(va, res[2])
    np.savez_compressed(os.path.join(HERE, "reference_ingest.npz"), **arr)
    with open(os.path.join(HERE, "reference_ingest.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", len(meta), "ingestion cases")


def make_matfree() -> None:
    """What the reference's matrix-free example prints (example/TestMatFree.cxx, built from
    the reference sources into oracle/_ref/test_matfree by build_ref.sh): per mesh dim
    (16, 32, ..., 512), the CG iteration count, the final residual norms and the L2 error."""
    import re
    import subprocess
    import tempfile
    O.build(ref=True)
    exe = os.path.join(ROOT, "oracle", "_ref", "test_matfree")
    with tempfile.TemporaryDirectory() as d:
        out = subprocess.run([exe], cwd=d, capture_output=True, text=True, check=True).stdout
    runs = {}
    for block in out.split("dim = ")[1:]:
        dim = int(block.split(",")[0])
        get = lambda key: re.search(key + r"\s*:\s*([-+0-9.eE]+)", block).group(1)  # noqa: E731
        runs[str(dim)] = dict(iters=int(get("NumIter")), norm2=get("Norm2"),
                              normInf=get("NormInf"), l2err=get("Error in L2-norm"))
    with open(os.path.join(HERE, "reference_matfree.json"), "w") as f:
        json.dump(runs, f, indent=1)
    print("wrote", len(runs), "matrix-free runs")


def mult_cases():
    """(name, L, R) of the MAT::Mult fixtures: stencil products, rectangular random factors
    with unsorted rows, duplicate columns and empty rows, and a Galerkin triple product."""
    rng = np.random.default_rng(77)

    def rand(n, m, per_row, empty=0.1):
        rp, ci, va = [0], [], []
        for i in range(n):
            if rng.random() >= empty:
                k = int(rng.integers(1, per_row + 1))
                cols = list(rng.integers(0, m, size=k))   # unsorted, may repeat
                ci += cols
                va += list(rng.integers(-8, 9, size=k) / 4.0 + rng.standard_normal(k) * 1e-3)
            rp.append(len(ci))
        return P.CSRMatrix(n, m, np.array(rp, np.uint32), np.array(ci, np.uint32),
                           np.array(va, np.float64))

    def interp1d(nf):
        nc = (nf - 1) // 2
        rp, ci, va = [0], [], []
        for i in range(nf):
            if i % 2 == 1:
                ci.append((i - 1) // 2)
                va.append(1.0)
            else:
                if i // 2 - 1 >= 0:
                    ci.append(i // 2 - 1)
                    va.append(0.5)
                if i // 2 < nc:
                    ci.append(i // 2)
                    va.append(0.5)
            rp.append(len(ci))
        return P.CSRMatrix(nf, nc, np.array(rp, np.uint32), np.array(ci, np.uint32),
                           np.array(va, np.float64))

    A = P.poisson2d(6)
    out = [("poisson2d_squared", A, A),
           ("random_rect", rand(20, 15, 5), rand(15, 25, 6)),
           ("random_dense_rows", rand(12, 40, 30, 0.0), rand(40, 9, 4))]
    Pm = interp1d(15)
    A1 = P.poisson2d(15, 1)
    Rt = P.CSRMatrix(Pm.mcol, Pm.nrow, *O.transpose("ref", Pm)[:3])
    out.append(("interp_R_times_A", Rt, A1))
    return out


def add_cases():
    """(name, a, A, b, B) of the MAT::Add fixtures: a stencil plus a shifted diagonal, random
    unsorted rows with repeated columns (row 0 starts with its smallest column: the
    reference's SortCSRRow cannot move an entry to the front of row 0), and B entries that
    repeat a column first appended from B (the one extra slot MAT::Add searches)."""
    rng = np.random.default_rng(91)

    def rand(n, m, per):
        rp, ci, va = [0], [], []
        for i in range(n):
            k = int(rng.integers(1, per + 1))
            cols = [0] if i == 0 else []
            cols += list(rng.integers(1 if i == 0 else 0, m, size=k))
            ci += cols
            va += list(rng.integers(-8, 9, size=len(cols)) / 8.0 + rng.standard_normal(len(cols)) * 1e-3)
            rp.append(len(ci))
        return P.CSRMatrix(n, m, np.array(rp, np.uint32), np.array(ci, np.uint32),
                           np.array(va, np.float64))

    A = P.poisson2d(6)
    D = P.CSRMatrix(36, 36, np.arange(37, dtype=np.uint32), np.arange(36, dtype=np.uint32),
                    np.linspace(0.5, 2.0, 36))
    # B rows that append a new column and then repeat it
    B3rp, B3ci, B3va = [0], [], []
    for i in range(36):
        cols = [0, (i + 7) % 36, (i + 7) % 36, (i + 9) % 36, (i + 7) % 36]
        B3ci += cols
        B3va += [0.25, 1.5, -0.75, 2.0, 0.125]
        B3rp.append(len(B3ci))
    B3 = P.CSRMatrix(36, 36, np.array(B3rp, np.uint32), np.array(B3ci, np.uint32),
                     np.array(B3va, np.float64))
    return [("stencil_plus_diag", 1.0, A, 0.5, D),
            ("random_unsorted", 0.5, rand(30, 20, 6), -1.25, rand(30, 20, 6)),
            ("repeated_appends", 2.0, A, -1.0, B3)]


def make_mult() -> None:
    O.build(ref=True)
    arr, meta = {}, {}
    for name, L, R in mult_cases():
        rp, ci, va = O.mat_mult("ref", L, R)
        for tag, M in (("L", L), ("R", R)):
            arr[f"{name}__{tag}_rowPtr"] = M.rowPtr
            arr[f"{name}__{tag}_colInd"] = M.colInd
            arr[f"{name}__{tag}_values"] = M.values
            meta[f"{name}__{tag}"] = [int(M.nrow), int(M.mcol)]
        arr[name + "__C_rowPtr"], arr[name + "__C_colInd"], arr[name + "__C_values"] = rp, ci, va
    for name, a, A, b, B in add_cases():
        code, (rp, ci, va) = O.mat_add("ref", a, A, b, B)
        assert code == 0, name
        for tag, M in (("A", A), ("B", B)):
            arr[f"add_{name}__{tag}_rowPtr"] = M.rowPtr
            arr[f"add_{name}__{tag}_colInd"] = M.colInd
            arr[f"add_{name}__{tag}_values"] = M.values
        meta[f"add_{name}"] = {"a": a, "b": b, "shape": [int(A.nrow), int(A.mcol)]}
        arr[f"add_{name}__C_rowPtr"], arr[f"add_{name}__C_colInd"] = rp, ci
        arr[f"add_{name}__C_values"] = va
    np.savez_compressed(os.path.join(HERE, "reference_mult.npz"), **arr)
    with open(os.path.join(HERE, "reference_mult.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", len(mult_cases()), "MAT::Mult and", len(add_cases()), "MAT::Add cases")


def make_mta() -> None:
    """MAT::MultTransposeAdd run by the reference on the cases' matrices."""
    O.build(ref=True)
    arr, meta = {}, {}
    for name, A in G.mta_matrices().items():
        v1, v2 = G.mta_vectors(A)
        code, v = O.mult_transpose_add("ref", A, v1, v2)
        assert code == 0, name
        trp, _, _, _ = O.transpose("port", A)
        arr[name + "__v"] = v
        meta[name] = {"symmetric_structure": bool(np.array_equal(trp, A.rowPtr))}
    np.savez_compressed(os.path.join(HERE, "reference_mta.npz"), **arr)
    with open(os.path.join(HERE, "reference_mta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", len(meta), "MAT::MultTransposeAdd cases")


if __name__ == "__main__":
    if "--mta-only" in sys.argv:
        make_mta()
        sys.exit(0)
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = args[0] if args else os.environ.get("FASPXX_REFERENCE")
    if not root or not os.path.isdir(os.path.join(root, "src")):
        sys.exit("make_golden.py: give the reference source tree as the first argument or "
                 "in FASPXX_REFERENCE")
    if "--mult-only" in sys.argv:
        make_mult()
        sys.exit(0)
    if "--runs-only" in sys.argv:  # the solver runs and transposes only
        main(root)
        sys.exit(0)
    if "--ingest-only" not in sys.argv and "--matfree-only" not in sys.argv:
        main(root)
    if "--matfree-only" not in sys.argv:
        make_ingest(root)
    make_matfree()
    make_mult()
    make_mta()
