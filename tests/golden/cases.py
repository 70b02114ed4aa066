"""Solver configurations replayed against the reference's recorded outputs.

Each case names a matrix (a bundled reference file or a seeded synthetic problem), the
right-hand side and initial guess, and the solver parameters of the reference example it
follows. ``make_golden.py`` records the compiled reference's results for these cases; the
CPU tests replay them on the C restatement and the GPU tests on the CUDA library.
"""
from __future__ import annotations

import os

import numpy as np

from faspxx_b200 import problems as P

HERE = os.path.dirname(os.path.abspath(__file__))

# data/input.param, the parameter file the reference examples read by default.
INPUT_PARAM = dict(maxIter=150, minIter=10, relTol=1e-5, absTol=1e-7)

# Known answers from the reference's unit tests.
# utest/src/UnitTestsMAT.cxx:42-46,64-67: mat1 * (0.314,...) == (0.314,2.826,2.512,0.942), TOL 1e-14.
MAT1 = dict(values=[0, 1, 2, 3, 4, 5, 2, 1, 2, 1], colInd=[0, 2, 0, 1, 3, 0, 2, 3, 2, 3],
            rowPtr=[0, 2, 5, 8, 10], x=[0.314] * 4, y=[0.314, 2.826, 2.512, 0.942], tol=1e-14)
# utest/src/UnitTestsJacobi.cxx:25-72 (2x2) and :75-156 (3x3), octave solutions, TOL 1e-5,
# weights 1.0 and 0.5; example/TestWeightedJacobi.cxx also uses 0.5 and 0.7.
JACOBI2 = dict(values=[4, 2, 1, 7], colInd=[0, 1, 0, 1], rowPtr=[0, 2, 4], b=[1, 1],
               xstar=[0.19231, 0.11538], tol=1e-5)
JACOBI3 = dict(values=[4, 2, 1, 3, 8, 2, 2, 1, 9], colInd=[0, 1, 2, 0, 1, 2, 0, 1, 2],
               rowPtr=[0, 3, 6, 9], b=[1, 1, 1], xstar=[0.221719, 0.027149, 0.058824], tol=1e-5)


def small_csr(d) -> P.CSRMatrix:
    n = len(d["rowPtr"]) - 1
    return P.CSRMatrix(n, n, np.array(d["rowPtr"], np.uint32), np.array(d["colInd"], np.uint32),
                       np.array(d["values"], np.float64))


_MAT_CACHE: dict = {}


def matrix(name: str) -> P.CSRMatrix:
    if name in _MAT_CACHE:
        return _MAT_CACHE[name]
    if name in ("fdm_10X10", "fem_small"):
        z = np.load(os.path.join(HERE, name + ".npz"))
        A = P.CSRMatrix(len(z["rowPtr"]) - 1, len(z["rowPtr"]) - 1, z["rowPtr"], z["colInd"],
                        z["values"])
    elif name == "poisson2d_32":
        A = P.poisson2d(32)
    elif name == "poisson3d_12":
        A = P.poisson3d(12)
    elif name == "convdiff_pe01":
        A = P.convdiff3d(10, 0.1)
    elif name == "convdiff_pe10":
        A = P.convdiff3d(10, 10.0)
    elif name == "vardiff_8":
        kappa = np.exp(np.random.default_rng(7).standard_normal(8 ** 3))
        A = P.vardiff3d(8, kappa)
    elif name == "jacobi2":
        A = small_csr(JACOBI2)
    elif name == "jacobi3":
        A = small_csr(JACOBI3)
    else:
        raise KeyError(name)
    _MAT_CACHE[name] = A
    return A


def case_inputs(case):
    A = matrix(case["mat"])
    n = A.nrow
    rhs = case.get("rhs", "zero")
    if rhs == "zero":
        b = np.zeros(n)
    elif rhs == "ones":
        b = np.ones(n)
    elif rhs == "xstar01":            # b = A x*, x* ~ U[0,1)
        b = A.matvec(P.seeded_uniform(n, 42))
    elif rhs == "xstar11":            # b = A x*, x* ~ U[-1,1)
        b = A.matvec(P.seeded_uniform(n, 42, -1.0, 1.0))
    elif rhs == "normal":
        b = np.random.default_rng(11).standard_normal(n)
    else:
        raise KeyError(rhs)
    x0 = np.ones(n) if case.get("x0", "ones") == "ones" else np.zeros(n)
    return A, b, x0


def solver_cases():
    C = []
    ip = INPUT_PARAM
    jac08 = dict(pcd="jacobi", pcdWeight=0.8, pcdIter=1)
    jac23 = dict(pcd="jacobi", pcdWeight=2.0 / 3.0, pcdIter=1)
    # example/TestPCG.cxx: weighted Jacobi 0.8, b = 0, x0 = 1
    C.append(dict(name="fdm_pcg", mat="fdm_10X10", alg="cg", kw=dict(**ip, **jac08)))
    C.append(dict(name="fdm_pcg_2sweeps", mat="fdm_10X10", alg="cg",
                  kw=dict(**ip, pcd="jacobi", pcdWeight=0.8, pcdIter=2)))
    # example/TestKrylov.cxx: Krylov() with the identity preconditioner
    for alg in ("cg", "bicgstab", "gmres", "gmres_left", "fgmres"):
        C.append(dict(name=f"fdm_{alg}", mat="fdm_10X10", alg=alg, kw=dict(ip)))
    # example/TestMG.cxx: 3 coarse levels of Jacobi smoothers, identity transfers
    C.append(dict(name="fdm_mg", mat="fdm_10X10", alg="mg", kw=dict(ip)))
    C.append(dict(name="fdm_mg_w", mat="fdm_10X10", alg="mg", kw=dict(ip, mgCycles=2)))
    C.append(dict(name="fdm_jacobi", mat="fdm_10X10", alg="jacobi", kw=dict(ip, weight=0.8)))
    # example/TestCG.cxx on fem_small (maxIter 500, relTol 1e-6)
    fem = dict(maxIter=500, minIter=0, relTol=1e-6, absTol=1e-8)
    for alg in ("cg", "bicgstab"):
        C.append(dict(name=f"fem_{alg}", mat="fem_small", alg=alg, kw=dict(fem)))
    C.append(dict(name="fem_pcg", mat="fem_small", alg="cg", kw=dict(fem, **jac08)))
    C.append(dict(name="fem_bicgstab_jac", mat="fem_small", alg="bicgstab", kw=dict(fem, **jac23)))
    for alg in ("gmres", "gmres_left", "fgmres"):
        C.append(dict(name=f"fem_{alg}_jac", mat="fem_small", alg=alg, kw=dict(fem, **jac23)))
        C.append(dict(name=f"fem_{alg}_jac_m30", mat="fem_small", alg=alg,
                      kw=dict(fem, **jac23, maxRestart=30, minRestart=30)))
    # FGMRES leaves Z[j] un-zeroed (FGMRES.cxx:158-159): with two Jacobi sweeps the
    # preconditioner warm-starts, also across two consecutive solves on one object.
    C.append(dict(name="fem_fgmres_jac2", mat="fem_small", alg="fgmres", repeat=2,
                  kw=dict(fem, pcd="jacobi", pcdWeight=2.0 / 3.0, pcdIter=2)))
    # CG quirks: minIter > 0 (denAbs = 1 while checking), and a tolerance below rounding
    # that drives the false-convergence restarts to ERROR_SOLVER_TOLSMALL (CG.cxx:186-215).
    C.append(dict(name="fdm_cg_min5", mat="fdm_10X10", alg="cg",
                  kw=dict(maxIter=100, minIter=5, relTol=1e-8, absTol=1e-12)))
    C.append(dict(name="fdm_cg_tolsmall", mat="fdm_10X10", alg="cg", rhs="ones",
                  kw=dict(maxIter=400, minIter=0, relTol=1e-17, absTol=0.0, restart=5)))
    C.append(dict(name="fdm_bicgstab_tolsmall", mat="fdm_10X10", alg="bicgstab", rhs="ones",
                  kw=dict(maxIter=400, minIter=0, relTol=1e-17, absTol=0.0, restart=5)))
    # The known-answer Jacobi systems (weights 1.0, 0.5, 0.7), solved as in the unit tests.
    for mname in ("jacobi2", "jacobi3"):
        for w in (1.0, 0.5, 0.7):
            C.append(dict(name=f"{mname}_w{w}", mat=mname, alg="jacobi", rhs="ones", x0="zero",
                          kw=dict(maxIter=100, relTol=1e-9, weight=w)))
    # Small synthetic versions of the benchmark workloads (b = A x*, x0 = 0).
    syn = dict(maxIter=2000, minIter=0, relTol=1e-8, absTol=0.0)
    C.append(dict(name="p2d_pcg", mat="poisson2d_32", alg="cg", rhs="xstar01", x0="zero",
                  store_b=True, kw=dict(syn, pcd="jacobi", pcdWeight=1.0, pcdIter=1)))
    C.append(dict(name="p3d_cg", mat="poisson3d_12", alg="cg", rhs="xstar01", x0="zero",
                  store_b=True, kw=dict(syn)))
    for pe in ("pe01", "pe10"):
        for alg in ("bicgstab", "gmres", "fgmres"):
            kw = dict(syn, **jac23)
            if alg != "bicgstab":
                kw.update(restart=30, maxRestart=30, minRestart=30)
            C.append(dict(name=f"cd_{pe}_{alg}", mat=f"convdiff_{pe}", alg=alg, rhs="xstar11",
                          x0="zero", store_b=True, kw=kw))
    C.append(dict(name="vd_cg", mat="vardiff_8", alg="cg", rhs="normal", x0="zero", store_b=True,
                  kw=dict(maxIter=2000, minIter=0, relTol=1e-10, absTol=0.0)))
    # The save branch taken in most iterations (savIter small: BiCGStab.cxx:133, CG.cxx's
    # safe copy): the iteration goes on after it with its direction update, and the saved x
    # is returned when numIter > savIter.
    C.append(dict(name="cd_pe01_bicgstab_sav3", mat="convdiff_pe01", alg="bicgstab",
                  rhs="xstar11", x0="zero", store_b=True, kw=dict(syn, **jac23, savIter=3)))
    C.append(dict(name="fdm_bicgstab_sav2", mat="fdm_10X10", alg="bicgstab",
                  kw=dict(ip, savIter=2)))
    C.append(dict(name="p2d_pcg_sav3", mat="poisson2d_32", alg="cg", rhs="xstar01", x0="zero",
                  store_b=True, kw=dict(syn, pcd="jacobi", pcdWeight=1.0, pcdIter=1,
                                        savIter=3)))
    # GMRES and FGMRES take it once per restart cycle (GMRES.cxx, FGMRES.cxx): restart 10
    for alg in ("gmres", "fgmres"):
        C.append(dict(name=f"cd_pe01_{alg}_sav3", mat="convdiff_pe01", alg=alg, rhs="xstar11",
                      x0="zero", store_b=True,
                      kw=dict(syn, **jac23, savIter=3, restart=10, maxRestart=10,
                              minRestart=10)))
    return C


def transpose_cases():
    return [("fdm_10X10", matrix("fdm_10X10")), ("fem_small", matrix("fem_small")),
            ("convdiff_pe10", matrix("convdiff_pe10")), ("jacobi3", matrix("jacobi3"))]


# ---- ReadMat conversions (reference_ingest.npz / .json, written by make_golden.py) ----------

_INGEST: dict = {}


def ingest_cases() -> dict:
    """name -> dict(kind, nrow, mcol, code, nnz, inputs=(a, b, values), expected=(rowPtr,
    colInd, values) or None when the reference leaves the MAT empty)."""
    if _INGEST:
        return _INGEST
    import json
    meta = json.load(open(os.path.join(HERE, "reference_ingest.json")))
    z = np.load(os.path.join(HERE, "reference_ingest.npz"))
    for name, m in meta.items():
        d = dict(m)
        d["inputs"] = (z[name + "__in0"], z[name + "__in1"], z[name + "__in2"])
        d["expected"] = ((z[name + "__rowPtr"], z[name + "__colInd"], z[name + "__values"])
                         if m["nnz"] else None)
        _INGEST[name] = d
    return _INGEST


def write_mtx(path: str, nrow: int, mcol: int, ri, ci, va) -> None:
    """MatrixMarket text of 0-based triplets (1-based in the file), values in repr form."""
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{nrow} {mcol} {len(va)}\n")
        for i, j, v in zip(ri, ci, va):
            f.write(f"{int(i) + 1} {int(j) + 1} {float(v)!r}\n")


def write_csr(path: str, n: int, rp, ci, va) -> None:
    """The text CSR layout ReadCSR reads: n, rowPtr, colInd, values, one number per line."""
    with open(path, "w") as f:
        f.write(f"{n}\n")
        for a in (rp, ci):
            f.write("".join(f"{int(x)}\n" for x in a))
        f.write("".join(f"{float(x)!r}\n" for x in va))


# ---- MAT::Mult (reference_mult.npz / .json, written by make_golden.py) ---------------------

def mult_cases() -> dict:
    """name -> (L, R, (rowPtr, colInd, values) of the reference's L R)."""
    import json
    from faspxx_b200 import problems as P
    meta = json.load(open(os.path.join(HERE, "reference_mult.json")))
    z = np.load(os.path.join(HERE, "reference_mult.npz"))
    out = {}
    for name in sorted({k.split("__")[0] for k in meta if not k.startswith("add_")}):
        mats = []
        for tag in ("L", "R"):
            nr, nc = meta[f"{name}__{tag}"]
            mats.append(P.CSRMatrix(nr, nc, z[f"{name}__{tag}_rowPtr"],
                                    z[f"{name}__{tag}_colInd"], z[f"{name}__{tag}_values"]))
        out[name] = (mats[0], mats[1], (z[name + "__C_rowPtr"], z[name + "__C_colInd"],
                                        z[name + "__C_values"]))
    return out


def add_cases() -> dict:
    """name -> (a, A, b, B, (rowPtr, colInd, values) of the reference's a A + b B)."""
    import json
    from faspxx_b200 import problems as P
    meta = json.load(open(os.path.join(HERE, "reference_mult.json")))
    z = np.load(os.path.join(HERE, "reference_mult.npz"))
    out = {}
    for key, m in meta.items():
        if not key.startswith("add_"):
            continue
        nr, nc = m["shape"]
        A, B = (P.CSRMatrix(nr, nc, z[f"{key}__{t}_rowPtr"], z[f"{key}__{t}_colInd"],
                            z[f"{key}__{t}_values"]) for t in ("A", "B"))
        out[key[4:]] = (m["a"], A, m["b"], B, (z[key + "__C_rowPtr"], z[key + "__C_colInd"],
                                                  z[key + "__C_values"]))
    return out


# ---- MAT::MultTransposeAdd (reference_mta.npz / .json, written by make_golden.py) ----------

def mta_matrices():
    """name -> square matrix for MAT::MultTransposeAdd. The first five are structurally
    symmetric (A's row pointers equal its transpose's), where the reference's loop bound
    (MAT.cxx:603, A's rowPtr instead of the transpose's) is right; ``rand_nonsym`` is not,
    and there the reference's result is not A^T v1 + v2."""
    from faspxx_b200 import problems as P
    out = {name: matrix(name) for name in ("fdm_10X10", "fem_small", "poisson3d_12",
                                           "convdiff_pe10", "vardiff_8")}
    rng = np.random.default_rng(31)
    n = 40
    rows, cols = [], []
    for i in range(n):
        extra = rng.choice(n, size=int(rng.integers(0, 6)), replace=False)
        for j in sorted(set(extra.tolist()) | {i}):
            rows.append(i)
            cols.append(j)
    rows, cols = np.array(rows), np.array(cols)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    out["rand_nonsym"] = P.CSRMatrix(n, n, rp.astype(np.uint32), cols.astype(np.uint32),
                                     rng.standard_normal(len(cols)))
    return out


def mta_vectors(A, seed=3):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(A.nrow), rng.standard_normal(A.mcol)


def mta_cases() -> dict:
    """name -> (A, v1, v2, the reference's v, structurally symmetric?)."""
    import json
    meta = json.load(open(os.path.join(HERE, "reference_mta.json")))
    z = np.load(os.path.join(HERE, "reference_mta.npz"))
    mats = mta_matrices()
    out = {}
    for name, m in meta.items():
        A = mats[name]
        v1, v2 = mta_vectors(A)
        out[name] = (A, v1, v2, z[name + "__v"], m["symmetric_structure"])
    return out


# ---- faults on the host side: bad inputs the solvers must report, not hang on -------------

def fault_cases():
    """name -> (alg, solver keywords, A, b, x0, compare x?) for the inputs CG.cxx:105-119,
    BiCGStab.cxx:118-124 and Iter.cxx:29-53 meet with NaN/Inf, a zero diagonal, maxIter = 1,
    a zero right-hand side and a zero matrix (every dot zero: the breakdown branches). The
    reference's own outcome on each is recorded by running it (tests/test_faults_cpu.py);
    x is compared only where the reference defines it (its CG breakdown reads an
    uninitialised alpha)."""
    from faspxx_b200 import problems as P
    A = matrix("fdm_10X10")
    n = A.nrow
    rng = np.random.default_rng(1)
    b = A.matvec(rng.random(n))
    bnan, binf = b.copy(), b.copy()
    bnan[5], binf[5] = np.nan, np.inf
    x0nan = np.zeros(n)
    x0nan[3] = np.nan
    vals = A.values.copy()
    vals[A.diag_ptr()[7]] = 0.0
    Azd = P.CSRMatrix(n, n, A.rowPtr, A.colInd, vals)
    Az0 = P.CSRMatrix(n, n, A.rowPtr, A.colInd, np.zeros(A.nnz))
    base = dict(maxIter=100, minIter=0, relTol=1e-8, absTol=0.0)
    out = {}
    for alg in ("cg", "bicgstab", "gmres", "fgmres"):
        for pname, pkw in (("id", {}), ("jac", dict(pcd="jacobi", pcdWeight=1.0, pcdIter=1))):
            kw = dict(base, **pkw)
            faults = [("nan_b", A, bnan, np.zeros(n)), ("inf_b", A, binf, np.zeros(n)),
                      ("nan_x0", A, b, x0nan), ("b0_x0", A, np.zeros(n), np.zeros(n))]
            if pkw:  # a zero diagonal is a fault only where Jacobi inverts it (Iter.cxx:45-47)
                faults.append(("zero_diag", Azd, b, np.zeros(n)))
            for tag, M, bb, x0 in faults:
                out[f"{alg}_{pname}_{tag}"] = (alg, kw, M, bb, x0, True)
            out[f"{alg}_{pname}_maxit1"] = (alg, dict(kw, maxIter=1), A, b, np.zeros(n), True)
        out[f"{alg}_zero_matrix"] = (alg, dict(base), Az0, np.ones(n), np.zeros(n),
                                     alg not in ("cg", "bicgstab"))
    return out
