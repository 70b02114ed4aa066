"""CPU ORACLE loader -- test infrastructure only.

Loads one of the two CPU back ends that share fasp_oracle.h:

* ``port`` -- ``liboracle_port.so``, the plain-C restatement (fasp_oracle.c);
* ``ref``  -- ``_ref/liboracle_ref.so``, the FASP++ sources compiled from their own tree
  by build_ref.sh, with the shim in ref_shim.cxx.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py`` (CPU baseline and reference arm)
import this module, as the checker or the timed CPU baseline. The GPU library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle_port.so")
REF_SO = os.path.join(HERE, "_ref", "liboracle_ref.so")

# Solver kinds (fasp_oracle.h; SOLType numbers, src/Param.hxx:36-54).
IDENTITY, CG, BICGSTAB, GMRES, FGMRES, JACOBI, MG, GMRES_LEFT = 0, 1, 2, 4, 5, 11, 21, 104
ALG_BY_NAME = {"cg": CG, "bicgstab": BICGSTAB, "gmres": GMRES, "fgmres": FGMRES,
               "jacobi": JACOBI, "mg": MG, "gmres_left": GMRES_LEFT}


class Params(C.Structure):
    _fields_ = [("maxIter", C.c_uint32), ("minIter", C.c_uint32), ("savIter", C.c_uint32),
                ("restart", C.c_uint32), ("relTol", C.c_double), ("absTol", C.c_double)]


class Config(C.Structure):
    _fields_ = [("alg", C.c_int), ("prm", Params), ("weight", C.c_double),
                ("maxRestart", C.c_uint32), ("minRestart", C.c_uint32),
                ("pcd", C.c_int), ("pcdWeight", C.c_double), ("pcdPrm", Params),
                ("mgLevels", C.c_uint32), ("mgCycles", C.c_uint32),
                ("mgSmoothWeight", C.c_double), ("mgCoarseWeight", C.c_double),
                ("mgSmoothPrm", Params), ("mgCoarsePrm", Params)]


_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compile the restatement and, with ref=True, the reference (build_ref.sh finds the
    reference tree from FASPXX_REFERENCE or its own default and skips when it is absent)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle_port.so"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


_LIBS: dict = {}


def load(kind: str = "port") -> C.CDLL:
    if kind in _LIBS:
        return _LIBS[kind]
    path = PORT_SO if kind == "port" else REF_SO
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library {path} is not built")
    lib = C.CDLL(path)
    lib.orc_default_params.argtypes = [C.POINTER(Params)]
    lib.orc_default_config.argtypes = [C.POINTER(Config), C.c_int]
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.POINTER(Config), C.c_uint32, C.c_uint32, C.c_uint32,
                               _u32p, _u32p, C.c_void_p]
    lib.orc_solve.restype = C.c_int
    lib.orc_solve.argtypes = [C.c_void_p, _f64p, _f64p, C.POINTER(C.c_uint32),
                              C.POINTER(C.c_double), C.POINTER(C.c_double), _f64p, C.c_uint32]
    lib.orc_clean.argtypes = [C.c_void_p]
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_spmv.argtypes = [C.c_uint32, _u32p, _u32p, C.c_void_p, _f64p, _f64p]
    lib.orc_residual.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _f64p, _f64p, _f64p,
                                 _f64p]
    for f in ("orc_dot",):
        getattr(lib, f).restype = C.c_double
        getattr(lib, f).argtypes = [C.c_uint32, _f64p, _f64p]
    for f in ("orc_norm2", "orc_norminf"):
        getattr(lib, f).restype = C.c_double
        getattr(lib, f).argtypes = [C.c_uint32, _f64p]
    lib.orc_transpose.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, _u32p, _u32p, C.c_void_p,
                                  _u32p, _u32p, C.c_void_p, C.c_void_p]
    lib.orc_diagptr.argtypes = [C.c_uint32, _u32p, _u32p, _u32p]
    lib.orc_mtx_to_mat.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, _u32p, _u32p, _f64p,
                                   C.POINTER(C.c_uint32), _u32p, _u32p, _f64p]
    lib.orc_csr_to_mat.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _f64p,
                                   C.POINTER(C.c_uint32), _u32p, _u32p, _f64p]
    _LIBS[kind] = lib
    return lib


def _vptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class Result:
    code: int
    x: np.ndarray
    iters: int
    norm2: float
    normInf: float
    hist: np.ndarray = field(repr=False)


def make_config(lib, alg: str, maxIter=1, minIter=0, savIter=100000, restart=30, relTol=1e-6,
                absTol=1e-8, weight=1.0, maxRestart=0, minRestart=0, pcd=None, pcdWeight=1.0,
                pcdIter=1, pcdMinIter=None, pcdRelTol=1e-6, pcdAbsTol=1e-8, mgLevels=3,
                mgCycles=1, mgSmooth=None, mgCoarse=None) -> Config:
    cfg = Config()
    lib.orc_default_config(C.byref(cfg), ALG_BY_NAME[alg])
    cfg.prm.maxIter, cfg.prm.minIter, cfg.prm.savIter = maxIter, minIter, savIter
    cfg.prm.restart, cfg.prm.relTol, cfg.prm.absTol = restart, relTol, absTol
    cfg.weight = weight
    cfg.maxRestart, cfg.minRestart = maxRestart, minRestart
    cfg.pcd = {"jacobi": 1, "mg": 2}.get(pcd, 0)
    cfg.pcdWeight = pcdWeight
    cfg.pcdPrm.maxIter = pcdIter
    cfg.pcdPrm.minIter = pcdIter if pcdMinIter is None else pcdMinIter
    cfg.pcdPrm.relTol, cfg.pcdPrm.absTol = pcdRelTol, pcdAbsTol
    cfg.mgLevels, cfg.mgCycles = mgLevels, mgCycles
    for name, spec in (("mgSmooth", mgSmooth), ("mgCoarse", mgCoarse)):
        if spec:
            prm = getattr(cfg, name + "Prm")
            for k, v in spec.items():
                if k == "weight":
                    setattr(cfg, name + "Weight", v)
                else:
                    setattr(prm, k, v)
    return cfg


class Solver:
    """One oracle solver object (the reference's Setup), reusable across solves."""

    def __init__(self, kind: str, mat, alg: str, **kw):
        self.lib = load(kind)
        self.cfg = make_config(self.lib, alg, **kw)
        rp, ci, va, n, m = mat.rowPtr, mat.colInd, mat.values, mat.nrow, mat.mcol
        self._keep = (rp, ci, va)
        self.n, self.m = n, m
        self.h = self.lib.orc_create(C.byref(self.cfg), n, m, len(ci), rp, ci, _vptr(va))
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        self.histCap = self.cfg.prm.maxIter + 2

    def solve(self, b, x0) -> Result:
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x0, dtype=np.float64, copy=True)
        hist = np.empty(self.histCap, dtype=np.float64)
        it, n2, ni = C.c_uint32(), C.c_double(), C.c_double()
        code = self.lib.orc_solve(self.h, b, x, C.byref(it), C.byref(n2), C.byref(ni), hist,
                                  self.histCap)
        return Result(code, x, it.value, n2.value, ni.value, hist[: it.value + 1].copy())

    def set_mg_level(self, level, P, R, Ac):
        """MG with transfer operators (port library): level's P, R and coarse operator."""
        self.lib.orc_mg_set_level.argtypes = [C.c_void_p, C.c_uint32] + \
            [C.c_uint32, C.c_uint32, C.c_uint32, _u32p, _u32p, _f64p] * 2 + \
            [C.c_uint32, C.c_uint32, _u32p, _u32p, _f64p]
        mats = []
        for M in (P, R, Ac):
            mats.append((np.ascontiguousarray(M.rowPtr, np.uint32),
                         np.ascontiguousarray(M.colInd, np.uint32),
                         np.ascontiguousarray(M.values, np.float64)))
        self._keep = self._keep + tuple(mats)
        (prp, pci, pva), (rrp, rci, rva), (arp, aci, ava) = mats
        code = self.lib.orc_mg_set_level(self.h, level, P.nrow, P.mcol, len(pci), prp, pci, pva,
                                         R.nrow, R.mcol, len(rci), rrp, rci, rva,
                                         Ac.nrow, len(aci), arp, aci, ava)
        assert code == 0, code

    def clean(self):
        self.lib.orc_clean(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None


def solve(kind, mat, alg, b, x0, **kw) -> Result:
    return Solver(kind, mat, alg, **kw).solve(b, x0)


def spmv(kind, mat, x):
    lib = load(kind)
    y = np.empty(mat.nrow, dtype=np.float64)
    lib.orc_spmv(mat.nrow, mat.rowPtr, mat.colInd, _vptr(mat.values),
                 np.ascontiguousarray(x, dtype=np.float64), y)
    return y


def residual(kind, mat, b, x):
    lib = load(kind)
    r = np.empty(mat.nrow, dtype=np.float64)
    lib.orc_residual(mat.nrow, mat.mcol, mat.rowPtr, mat.colInd, mat.values,
                     np.ascontiguousarray(b, np.float64), np.ascontiguousarray(x, np.float64), r)
    return r


def dot(kind, a, b):
    a = np.ascontiguousarray(a, np.float64)
    return load(kind).orc_dot(len(a), a, np.ascontiguousarray(b, np.float64))


def norm2(kind, a):
    a = np.ascontiguousarray(a, np.float64)
    return load(kind).orc_norm2(len(a), a)


def norminf(kind, a):
    a = np.ascontiguousarray(a, np.float64)
    return load(kind).orc_norminf(len(a), a)


def transpose(kind, mat):
    """MAT::TransInPlace: returns (rowPtr, colInd, values, diagPtr) of the transpose."""
    lib = load(kind)
    nnz = len(mat.colInd)
    trp = np.empty(mat.mcol + 1, np.uint32)
    tci = np.empty(nnz, np.uint32)
    tva = None if mat.values is None else np.empty(nnz, np.float64)
    tdp = np.empty(mat.mcol, np.uint32)
    lib.orc_transpose(mat.nrow, mat.mcol, nnz, mat.rowPtr, mat.colInd, _vptr(mat.values),
                      trp, tci, _vptr(tva), tdp.ctypes.data_as(C.c_void_p))
    return trp, tci, tva, tdp


# ORC_REF_UNDEFINED (fasp_oracle.h): the reference indexes out of bounds on this input.
REF_UNDEFINED = -1000


def mult_transpose_add(kind, mat, v1, v2):
    """MAT::MultTransposeAdd: (code, v = A^T v1 + v2); the reference back end returns
    REF_UNDEFINED (and no v) where its loop would read past A's row pointers."""
    lib = load(kind)
    lib.orc_mult_transpose_add.restype = C.c_int
    lib.orc_mult_transpose_add.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, C.c_void_p,
                                           _f64p, _f64p, _f64p]
    v = np.zeros(mat.mcol)
    code = lib.orc_mult_transpose_add(mat.nrow, mat.mcol, mat.rowPtr, mat.colInd,
                                      _vptr(mat.values), np.ascontiguousarray(v1, np.float64),
                                      np.ascontiguousarray(v2, np.float64), v)
    return code, (v if code == 0 else None)


def _converted(code, nnz_out, rp, ci, va):
    n = nnz_out.value
    return code, (rp, ci[:n].copy(), va[:n].copy()) if n else None


def mtx_to_mat(kind, nrow, mcol, rowInd, colInd, values):
    """MTXtoMAT of 0-based triplets: (code, (rowPtr, colInd, values) or None if empty)."""
    ri = np.ascontiguousarray(rowInd, np.uint32)
    ci = np.ascontiguousarray(colInd, np.uint32)
    va = np.ascontiguousarray(values, np.float64)
    cap = len(ci) + nrow
    rp_o, ci_o, va_o = np.zeros(nrow + 1, np.uint32), np.empty(cap, np.uint32), np.empty(cap)
    z = C.c_uint32()
    code = load(kind).orc_mtx_to_mat(nrow, mcol, len(ci), ri, ci, va, C.byref(z), rp_o, ci_o,
                                     va_o)
    return _converted(code, z, rp_o, ci_o, va_o)


def csr_to_mat(kind, nrow, rowPtr, colInd, values):
    """ReadMat's .csr conversions of raw (0- or 1-based) CSR arrays: (code, arrays or None)."""
    rp = np.ascontiguousarray(rowPtr, np.uint32)
    ci = np.ascontiguousarray(colInd, np.uint32)
    va = np.ascontiguousarray(values, np.float64)
    cap = len(ci) + nrow
    rp_o, ci_o, va_o = np.zeros(nrow + 1, np.uint32), np.empty(cap, np.uint32), np.empty(cap)
    z = C.c_uint32()
    code = load(kind).orc_csr_to_mat(nrow, len(ci), rp, ci, va, C.byref(z), rp_o, ci_o, va_o)
    return _converted(code, z, rp_o, ci_o, va_o)


def matfree_rhs(dim: int) -> np.ndarray:
    """The right-hand side of the reference's matrix-free example at mesh `dim` (port)."""
    lib = load("port")
    lib.orc_matfree_rhs.argtypes = [C.c_int, _f64p]
    b = np.empty((dim - 1) ** 2)
    lib.orc_matfree_rhs(dim, b)
    return b


def mat_mult(kind, L, R):
    """MAT::Mult: (rowPtr, colInd, values) of L R (CSRMatrix-like L and R)."""
    lib = load(kind)
    lib.orc_mat_mult.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, _f64p, C.c_uint32,
                                 _u32p, _u32p, _f64p, C.c_uint32, C.POINTER(C.c_uint32),
                                 _u32p, _u32p, _f64p]
    lrp, lci = np.ascontiguousarray(L.rowPtr, np.uint32), np.ascontiguousarray(L.colInd, np.uint32)
    rrp, rci = np.ascontiguousarray(R.rowPtr, np.uint32), np.ascontiguousarray(R.colInd, np.uint32)
    lva, rva = np.ascontiguousarray(L.values, np.float64), np.ascontiguousarray(R.values, np.float64)
    rlen = np.diff(rrp.astype(np.int64))
    cap = int(rlen[lci].sum()) if len(lci) else 0
    rp = np.zeros(L.nrow + 1, np.uint32)
    ci = np.empty(max(cap, 1), np.uint32)
    va = np.empty(max(cap, 1), np.float64)
    z = C.c_uint32()
    code = lib.orc_mat_mult(L.nrow, L.mcol, lrp, lci, lva, R.mcol, rrp, rci, rva, cap,
                            C.byref(z), rp, ci, va)
    assert code == 0
    return rp, ci[:z.value].copy(), va[:z.value].copy()


def mat_add(kind, a, A, b, B):
    """MAT::Add: (code, (rowPtr, colInd, values)) of a A + b B."""
    lib = load(kind)
    lib.orc_mat_add.argtypes = [C.c_uint32, C.c_uint32, C.c_double, _u32p, _u32p, _f64p,
                                C.c_double, _u32p, _u32p, _f64p, C.POINTER(C.c_uint32),
                                _u32p, _u32p, _f64p]
    arrs = [np.ascontiguousarray(x, t) for x, t in
            ((A.rowPtr, np.uint32), (A.colInd, np.uint32), (A.values, np.float64),
             (B.rowPtr, np.uint32), (B.colInd, np.uint32), (B.values, np.float64))]
    cap = len(arrs[1]) + len(arrs[4])
    rp = np.zeros(A.nrow + 1, np.uint32)
    ci, va = np.empty(max(cap, 1), np.uint32), np.empty(max(cap, 1), np.float64)
    z = C.c_uint32()
    code = lib.orc_mat_add(A.nrow, A.mcol, a, arrs[0], arrs[1], arrs[2], b, arrs[3], arrs[4],
                           arrs[5], C.byref(z), rp, ci, va)
    return code, (rp, ci[:z.value].copy(), va[:z.value].copy())
