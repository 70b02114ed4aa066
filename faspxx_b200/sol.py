"""Python mirror of the FASP++ solver API (MAT/VEC/LOP and the SOL family) over the C ABI.

Names, setters and return codes follow the reference (src/MAT.hxx, src/VEC.hxx,
src/SOL.hxx, src/CG.hxx, src/BiCGStab.hxx, src/GMRES.hxx, src/FGMRES.hxx, src/Iter.hxx,
src/MG.hxx) so that a driver written against the reference reads the same here:

    A = MAT(csr); pcd = Jacobi(); pcd.SetWeight(0.8); pcd.SetMaxIter(1); pcd.SetMinIter(1)
    pcd.Setup(A); solver = CG(); solver.SetMaxIter(200); solver.SetupPCD(pcd)
    solver.Setup(A); code = solver.Solve(b, x)        # x: initial guess in, solution out

``b``/``x`` may be NumPy arrays (host; the end-to-end path copies them) or ``DVec``
(device vectors already in HBM). Every operation runs on the GPU through libfasp_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import check, lib
from .problems import CSRMatrix

# Output levels of src/Param.hxx:27-33 (printing is the caller's business here).
PRINT_NONE, PRINT_MIN, PRINT_SOME, PRINT_MORE, PRINT_MAX = 0, 2, 4, 6, 8


class DVec:
    """A VEC resident in device memory (float64); DVec(n) holds n zeros, as VEC(size) does
    (src/VEC.hxx:43)."""

    def __init__(self, n: int, host: np.ndarray | None = None):
        capi.init()
        self.n = int(n)
        p = C.c_void_p()
        check(lib.fasp_gpu_malloc(C.byref(p), max(8, self.n * 8) + 16), "fasp_gpu_malloc")
        self.ptr = p
        if host is not None:
            self.set(host)
        else:
            self.Zero()

    def Zero(self) -> None:
        """Every entry 0.0 (a memset: unlike Scale(0.0), it also clears NaN and Inf)."""
        check(lib.fasp_gpu_memset(self.ptr, 0, max(8, self.n * 8)), "fasp_gpu_memset")

    @classmethod
    def from_numpy(cls, a) -> "DVec":
        a = np.ascontiguousarray(a, dtype=np.float64)
        return cls(a.shape[0], a)

    def set(self, a) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape[0] == self.n
        check(lib.fasp_gpu_memcpy_h2d(self.ptr, a.ctypes.data, self.n * 8), "h2d")

    def numpy(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(lib.fasp_gpu_memcpy_d2h(out.ctypes.data, self.ptr, self.n * 8), "d2h")
        return out

    def GetSize(self) -> int:
        return self.n

    # VEC members that the solvers use (src/VEC.cxx)
    def Dot(self, v: "DVec") -> float:
        r = C.c_double()
        check(lib.fasp_gpu_vec_dot(self.n, self.ptr, v.ptr, C.byref(r)), "Dot")
        return r.value

    def Norm2(self) -> float:
        r = C.c_double()
        check(lib.fasp_gpu_vec_norm2(self.n, self.ptr, C.byref(r)), "Norm2")
        return r.value

    def NormInf(self) -> float:
        r = C.c_double()
        check(lib.fasp_gpu_vec_norminf(self.n, self.ptr, C.byref(r)), "NormInf")
        return r.value

    def AXPY(self, a: float, x: "DVec") -> None:
        check(lib.fasp_gpu_vec_axpy(self.n, a, x.ptr, self.ptr), "AXPY")

    def XPAY(self, a: float, x: "DVec") -> None:
        check(lib.fasp_gpu_vec_xpay(self.n, a, x.ptr, self.ptr), "XPAY")

    def AXPBY(self, a: float, b: float, y: "DVec") -> None:
        check(lib.fasp_gpu_vec_axpby(self.n, a, b, y.ptr, self.ptr), "AXPBY")

    def WAXPBY(self, a: float, v1: "DVec", b: float, v2: "DVec") -> None:
        check(lib.fasp_gpu_vec_waxpby(self.n, a, v1.ptr, b, v2.ptr, self.ptr), "WAXPBY")

    def Scale(self, a: float) -> None:
        check(lib.fasp_gpu_vec_scale(self.n, a, self.ptr), "Scale")

    def __del__(self):
        if getattr(self, "ptr", None):
            lib.fasp_gpu_free(self.ptr)
            self.ptr = None


class MAT:
    """CSRx matrix in HBM (src/MAT.hxx)."""

    def __init__(self, csr: CSRMatrix | None = None, _handle=None):
        capi.init()
        self.h = None
        if _handle is not None:
            self.h = _handle
        elif csr is not None:
            h = C.c_void_p()
            rp = np.ascontiguousarray(csr.rowPtr, dtype=np.uint32)
            ci = np.ascontiguousarray(csr.colInd, dtype=np.uint32)
            va = None if csr.values is None else np.ascontiguousarray(csr.values, np.float64)
            check(lib.fasp_gpu_mat_create(csr.nrow, csr.mcol, len(ci), rp.ctypes.data,
                                          ci.ctypes.data,
                                          None if va is None else va.ctypes.data, C.byref(h)),
                  "MAT")
            self.h = h
        n, m, z = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib.fasp_gpu_mat_info(self.h, C.byref(n), C.byref(m), C.byref(z)), "info")
        self.nrow, self.mcol, self.nnz = n.value, m.value, z.value

    @classmethod
    def FromCOO(cls, nrow: int, mcol: int, rowInd, colInd, values) -> "MAT":
        """MTXtoMAT (src/MATUtil.cxx:416-436) on the GPU: 0-based triplets in any order,
        duplicates kept, rows sorted stably by column, missing diagonals stored as 0.0.
        The arrays are host NumPy arrays, or DVec-like objects with a device ``ptr``
        (row and column indices as uint32, values as float64)."""
        return cls._ingest(lib.fasp_gpu_mat_create_coo, "MTXtoMAT", nrow, mcol, _count(values),
                           rowInd, colInd, values)

    @classmethod
    def FromCSRRaw(cls, nrow: int, rowPtr, colInd, values, mcol: int | None = None) -> "MAT":
        """ReadMat's .csr conversions (src/ReadData.cxx:350-353,376-400) on the GPU: raw
        CSR arrays, 0- or 1-based, rows in any column order."""
        return cls._ingest(lib.fasp_gpu_mat_create_csr_raw, "ReadCSR", nrow,
                           nrow if mcol is None else mcol, _count(values), rowPtr, colInd,
                           values)

    @classmethod
    def Stencil(cls, shape, points) -> "MAT":
        """A matrix-free operator on a structured grid (the GPU form of the reference's
        matrix-free LOP, example/TestMatFree.cxx:26-176): shape = (nx,), (nx, ny) or
        (nx, ny, nz); points = [((dx, dy, dz), coef), ...] (shorter offset tuples are
        padded with 0). Row ix + nx (iy + ny iz); the stencil is truncated at the faces."""
        capi.init()
        dims = list(shape) + [1] * (3 - len(shape))
        off = [tuple(list(o) + [0] * (3 - len(o))) for o, _ in points]
        dx = np.array([o[0] for o in off], np.int32)
        dy = np.array([o[1] for o in off], np.int32)
        dz = np.array([o[2] for o in off], np.int32)
        cf = np.array([c for _, c in points], np.float64)
        h = C.c_void_p()
        check(lib.fasp_gpu_mat_create_stencil(dims[0], dims[1], dims[2], len(cf),
                                              dx.ctypes.data, dy.ctypes.data, dz.ctypes.data,
                                              cf.ctypes.data, C.byref(h)), "MatFree")
        return cls(_handle=h)

    @classmethod
    def _ingest(cls, fn, where, nrow, mcol, nnz, a, b, v) -> "MAT":
        capi.init()
        dev = hasattr(v, "ptr")
        if dev:
            ptrs = [x.ptr for x in (a, b, v)]
        else:
            keep = [np.ascontiguousarray(a, np.uint32), np.ascontiguousarray(b, np.uint32),
                    np.ascontiguousarray(v, np.float64)]
            ptrs = [x.ctypes.data for x in keep]
        h = C.c_void_p()
        check(fn(nrow, mcol, nnz, *ptrs, 1 if dev else 0, C.byref(h)), where)
        return cls(_handle=h)

    def GetRowSize(self) -> int:
        return self.nrow

    def GetColSize(self) -> int:
        return self.mcol

    def GetNNZ(self) -> int:
        return self.nnz

    def Apply(self, v: DVec, w: DVec) -> None:
        check(lib.fasp_gpu_mat_apply(self.h, v.ptr, w.ptr), "Apply")

    def Residual(self, b: DVec, x: DVec, r: DVec) -> None:
        check(lib.fasp_gpu_mat_residual(self.h, b.ptr, x.ptr, r.ptr), "Residual")

    def MultTransposeAdd(self, v1: DVec, v2: DVec, v: DVec) -> None:
        """MAT::MultTransposeAdd (src/MAT.cxx:541-606): v = A^T v1 + v2 on the cached exact
        transpose, in the reference's operation order."""
        check(lib.fasp_gpu_mat_mult_transpose_add(self.h, v1.ptr, v2.ptr, v.ptr),
              "MultTransposeAdd")

    def SetRowClass(self, mode) -> None:
        """Matrix form of the SpMV kernels: 0/False = CSR, 1 = row classes, 2/True = row
        classes with stencil masks (the default when built)."""
        mode = 2 if mode is True else (0 if mode is False else int(mode))
        check(lib.fasp_gpu_mat_set_rowclass(self.h, mode), "SetRowClass")

    def SetCol16(self, on: bool) -> None:
        """Use (True) or ignore (False, the default) the 16-bit column offsets."""
        check(lib.fasp_gpu_mat_set_col16(self.h, 1 if on else 0), "SetCol16")

    def Col16Info(self):
        """(built, in use) of the 16-bit column offsets."""
        b, u = C.c_int(), C.c_int()
        check(lib.fasp_gpu_mat_col16_info(self.h, C.byref(b), C.byref(u)), "Col16Info")
        return bool(b.value), bool(u.value)

    def TileInfo(self):
        """(span, fits FP64, fits FP32, CSR form with one thread per row in use) of the
        block tiles: the most entries a 256-row tile covers and whether every tile fits a
        stage; the tiles run where the form is in use and the tile fits."""
        sp, f64, f32, u = C.c_uint32(), C.c_int(), C.c_int(), C.c_int()
        check(lib.fasp_gpu_mat_tile_info(self.h, C.byref(sp), C.byref(f64), C.byref(f32),
                                         C.byref(u)), "TileInfo")
        return sp.value, bool(f64.value), bool(f32.value), bool(u.value)

    def RowClassInfo(self):
        """(mode in use, classes, table entries, stencil length); 0 classes: no row-class
        form, stencil 0: no masks."""
        mode, k, e, st = C.c_int(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib.fasp_gpu_mat_rowclass_info(self.h, C.byref(mode), C.byref(k), C.byref(e),
                                             C.byref(st)), "RowClassInfo")
        return mode.value, k.value, e.value, st.value

    def Mult(self, R: "MAT") -> "MAT":
        """MAT::Mult (src/MAT.cxx:715-800): self * R as a new matrix, computed on the GPU."""
        h = C.c_void_p()
        check(lib.fasp_gpu_mat_mult(self.h, R.h, C.byref(h)), "Mult")
        return MAT(_handle=h)

    @staticmethod
    def Add(a: float, A: "MAT", b: float, B: "MAT") -> "MAT":
        """MAT::Add (src/MAT.cxx:652-713): a A + b B as a new matrix, computed on the GPU."""
        h = C.c_void_p()
        check(lib.fasp_gpu_mat_add(a, A.h, b, B.h, C.byref(h)), "Add")
        return MAT(_handle=h)

    def Transpose(self) -> "MAT":
        """MAT::TransInPlace into a new matrix (the original stays)."""
        h = C.c_void_p()
        check(lib.fasp_gpu_mat_transpose(self.h, C.byref(h)), "TransInPlace")
        return MAT(_handle=h)

    def download(self) -> CSRMatrix:
        rp = np.empty(self.nrow + 1, np.uint32)
        ci = np.empty(self.nnz, np.uint32)
        va = np.empty(self.nnz, np.float64)
        check(lib.fasp_gpu_mat_download(self.h, rp.ctypes.data, ci.ctypes.data, va.ctypes.data,
                                        None), "download")
        return CSRMatrix(self.nrow, self.mcol, rp, ci, va)

    def diag_ptr(self) -> np.ndarray:
        dp = np.empty(self.nrow, np.uint32)
        check(lib.fasp_gpu_mat_download(self.h, None, None, None, dp.ctypes.data), "diagPtr")
        return dp

    def Autotune(self) -> int:
        L = C.c_int()
        check(lib.fasp_gpu_mat_autotune(self.h, C.byref(L)), "autotune")
        return L.value

    def SetLanes(self, lanes: int) -> None:
        check(lib.fasp_gpu_mat_set_lanes(self.h, lanes), "set_lanes")

    def SampledOuter(self, lam: DVec, x: DVec, scale: float, out: DVec) -> None:
        check(lib.fasp_gpu_mat_sampled_outer(self.h, lam.ptr, x.ptr, scale, out.ptr),
              "sampled_outer")

    def __del__(self):
        if getattr(self, "h", None):
            lib.fasp_gpu_mat_destroy(self.h)
            self.h = None


def tile_timeouts() -> int:
    """Block-tile waits that ran out since the library was loaded (0 on a healthy device)."""
    capi.init()
    c = C.c_uint32()
    check(lib.fasp_gpu_tile_timeouts(C.byref(c)), "tile_timeouts")
    return c.value


def _count(a) -> int:
    return int(a.n) if hasattr(a, "ptr") else len(a)


def ReadMat(path: str) -> MAT:
    """ReadMat (src/ReadData.cxx:361-446): a .csr or .mtx file by its extension. The text
    is parsed on the host (read_csr_raw / read_mtx_raw); sorting, the 1-based shift and
    the diagonal insertion run on the GPU. Unknown extension: ERROR_INPUT_FILE (-11)."""
    from .problems import read_csr_raw, read_mtx_raw
    ext = path[-3:].lower() if len(path) > 4 else ""
    if ext == "csr":
        n, rp, ci, va = read_csr_raw(path)
        return MAT.FromCSRRaw(n, rp, ci, va)
    if ext == "mtx":
        nrow, mcol, ri, ci, va = read_mtx_raw(path)
        return MAT.FromCOO(nrow, mcol, ri, ci, va)
    raise capi.FaspError(-11, "ReadMat")


class SOL:
    """Base solver (src/SOL.hxx:24-126); subclasses fix the algorithm."""

    ALG = capi.CG

    def __init__(self):
        capi.init()
        self.cfg = capi.default_config(self.ALG)
        self.A: MAT | None = None
        self.h = None
        self._built = None
        self.numIter = 0
        self.norm2 = 1e60
        self.normInf = 1e60
        self.info = capi.Info()

    # setters (src/SOL.cxx:102-124)
    def SetOutput(self, verbose):
        self.verbose = verbose

    def SetMaxIter(self, v):
        self.cfg.prm.maxIter = int(v)

    def SetMinIter(self, v):
        self.cfg.prm.minIter = int(v)

    def SetSavIter(self, v):
        self.cfg.prm.savIter = int(v)

    def SetRestart(self, v):
        self.cfg.prm.restart = int(v)

    def SetRelTol(self, v):
        self.cfg.prm.relTol = float(v)

    def SetAbsTol(self, v):
        self.cfg.prm.absTol = float(v)

    # B200 options
    def SetPrecision(self, p, innerRelTol=None, innerMaxIter=None, maxOuter=None):
        self.cfg.precision = p
        if innerRelTol is not None:
            self.cfg.innerRelTol = innerRelTol
        if innerMaxIter is not None:
            self.cfg.innerMaxIter = innerMaxIter
        if maxOuter is not None:
            self.cfg.maxOuter = maxOuter

    def SetOrth(self, orth):
        self.cfg.orth = orth

    def SetPersistent(self, flag):
        """False: CUDA graphs; True (1): one cooperative launch; 2: one thread-block cluster."""
        self.cfg.persistent = int(flag)

    def SetOverlapLaunch(self, flag: bool):
        self.cfg.overlapLaunch = 1 if flag else 0

    def SetFP32Recurrence(self, flag: bool):
        self.cfg.fp32Recurrence = 1 if flag else 0

    def SetUseGraph(self, flag: bool):
        self.cfg.useGraph = 1 if flag else 0

    def SetupPCD(self, pc: "SOL"):
        """SOL::SetupPCD (SOL.cxx:249): Identity or Jacobi, its weight and SOLParams."""
        if isinstance(pc, Jacobi):
            self.cfg.pcd = 1
            self.cfg.pcdWeight = pc.weight
            self.cfg.pcdPrm = capi.Params(pc.cfg.prm.maxIter, pc.cfg.prm.minIter,
                                          pc.cfg.prm.savIter, pc.cfg.prm.restart,
                                          pc.cfg.prm.relTol, pc.cfg.prm.absTol)
        elif isinstance(pc, Identity):
            self.cfg.pcd = 0
        elif isinstance(pc, MG):
            # MG as the preconditioner: its SOLParams, levels, cycles, smoother and coarse
            # solver settings and transfer operators
            self.cfg.pcd = 2
            p = pc.cfg.prm
            self.cfg.pcdPrm = capi.Params(p.maxIter, p.minIter, p.savIter, p.restart, p.relTol,
                                          p.absTol)
            for f in ("mgLevels", "mgCycles", "mgSmoothWeight", "mgCoarseWeight",
                      "mgSmoothPrm", "mgCoarsePrm"):
                setattr(self.cfg, f, getattr(pc.cfg, f))
            self.transfers = dict(getattr(pc, "transfers", {}))
            self._built = None
        else:
            raise capi.FaspError(-31, "SetupPCD")

    def Setup(self, A: MAT) -> int:
        self.A = A
        self._build()
        return 0

    def _key(self):
        return bytes(self.cfg)

    def _build(self):
        if self.A is None:
            raise capi.FaspError(-12, "Setup")
        if self.h is not None and self._built == self._key():
            return
        self._destroy()
        h = C.c_void_p()
        check(lib.fasp_gpu_solver_create(C.byref(self.cfg), C.byref(h)), "solver_create")
        self.h = h
        for level, (P, R, Ac) in sorted(getattr(self, "transfers", {}).items()):
            check(lib.fasp_gpu_solver_set_mg_transfer(self.h, level, P.h,
                                                      None if R is None else R.h,
                                                      None if Ac is None else Ac.h),
                  "set_mg_transfer")
        check(lib.fasp_gpu_solver_setup(self.h, self.A.h), "Setup")
        self._built = self._key()

    def Solve(self, b, x) -> int:
        """Solve(b, x); returns the FaspRetCode. x is updated in place."""
        self._build()
        if isinstance(b, DVec):
            code = lib.fasp_gpu_solver_solve(self.h, b.ptr, x.ptr, C.byref(self.info))
        else:
            bb = np.ascontiguousarray(b, dtype=np.float64)
            if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
                raise TypeError("x must be a contiguous float64 NumPy array or a DVec")
            code = lib.fasp_gpu_solver_solve_host(self.h, bb.ctypes.data, x.ctypes.data,
                                                  C.byref(self.info))
        if code not in (0,) and code <= -100:
            check(code, "Solve")
        self.numIter = self.info.numIter
        self.norm2 = self.info.norm2
        self.normInf = self.info.normInf
        return self.info.code if code == 0 else code

    def SolveAdjoint(self, g, lam) -> int:
        """Solve A^T lam = g with the same configuration (exact CSC transpose)."""
        self._build()
        code = lib.fasp_gpu_solver_solve_adjoint(self.h, g.ptr, lam.ptr, C.byref(self.info))
        if code <= -100:
            check(code, "SolveAdjoint")
        return self.info.code if code == 0 else code

    def GetIterations(self) -> int:
        return self.numIter

    def GetNorm2(self) -> float:
        return self.norm2

    def GetInfNorm(self) -> float:
        return self.normInf

    def History(self) -> np.ndarray:
        n = C.c_uint32()
        check(lib.fasp_gpu_solver_history(self.h, None, 0, C.byref(n)), "history")
        out = np.empty(n.value, np.float64)
        check(lib.fasp_gpu_solver_history(self.h, out.ctypes.data, n.value, C.byref(n)), "history")
        return out

    def LastTimeMs(self) -> float:
        t = C.c_double()
        check(lib.fasp_gpu_solver_last_time(self.h, C.byref(t)), "last_time")
        return t.value

    def Clean(self):
        if self.h is not None:
            check(lib.fasp_gpu_solver_clean(self.h), "Clean")

    def _destroy(self):
        if self.h is not None:
            lib.fasp_gpu_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        self._destroy()


class CG(SOL):
    ALG = capi.CG


class BiCGStab(SOL):
    ALG = capi.BICGSTAB


class GMRES(SOL):
    ALG = capi.GMRES

    def SetMaxMinRestart(self, maxRestart, minRestart):
        self.cfg.maxRestart, self.cfg.minRestart = int(maxRestart), int(minRestart)

    def SetRightPrecond(self):
        self.cfg.leftPrecond = 0

    def SetLeftPrecond(self):
        self.cfg.leftPrecond = 1


class FGMRES(SOL):
    ALG = capi.FGMRES

    def SetMaxMinRestart(self, maxRestart, minRestart):
        self.cfg.maxRestart, self.cfg.minRestart = int(maxRestart), int(minRestart)


class Identity(SOL):
    """Identity::Solve (Iter.cxx:16-20); only meaningful as a preconditioner."""
    ALG = capi.IDENTITY


class Jacobi(SOL):
    """Jacobi / weighted Jacobi (Iter.hxx:42-71)."""
    ALG = capi.JACOBI

    def __init__(self, weight: float = 1.0):
        super().__init__()
        self.weight = float(weight)
        self.cfg.weight = self.weight

    def SetWeight(self, w):
        self.weight = float(w)
        self.cfg.weight = self.weight


class MG(SOL):
    """Abstract MG with identity transfers and Jacobi smoothers/coarse solvers (MG.hxx), or,
    with SetTransfer for every coarse level, MG with restriction/prolongation operators and
    per-level operators (a B200 extension; see fasp_gpu_solver_set_mg_transfer)."""
    ALG = capi.MG

    def SetTransfer(self, level: int, P: MAT, R: MAT | None = None, Ac: MAT | None = None):
        """Level `level` (0 = finest): prolongation P from level+1, restriction R (None: P's
        transpose) and coarse operator Ac (None: the Galerkin product R A P on the GPU)."""
        if not hasattr(self, "transfers"):
            self.transfers = {}
        self.transfers[int(level)] = (P, R, Ac)
        self._built = None

    def SetupALL(self, A: MAT, numLevels: int):
        self.cfg.mgLevels = int(numLevels)
        self.A = A

    def SetNumCycles(self, ncycle: int):
        self.cfg.mgCycles = int(ncycle)

    def SetSmoother(self, weight=1.0, maxIter=1, minIter=0, relTol=1e-6, absTol=1e-8):
        self.cfg.mgSmoothWeight = weight
        self.cfg.mgSmoothPrm = capi.Params(maxIter, minIter, 100000, 30, relTol, absTol)

    def SetCoarseSolver(self, weight=1.0, maxIter=1, minIter=0, relTol=1e-6, absTol=1e-8):
        self.cfg.mgCoarseWeight = weight
        self.cfg.mgCoarsePrm = capi.Params(maxIter, minIter, 100000, 30, relTol, absTol)


ALG_CLASS = {"cg": CG, "bicgstab": BiCGStab, "gmres": GMRES, "gmres_left": GMRES,
             "fgmres": FGMRES, "jacobi": Jacobi, "mg": MG}


def configure(alg: str, maxIter=1, minIter=0, savIter=100000, restart=30, relTol=1e-6,
              absTol=1e-8, weight=1.0, maxRestart=0, minRestart=0, pcd=None, pcdWeight=1.0,
              pcdIter=1, pcdMinIter=None, pcdRelTol=1e-6, pcdAbsTol=1e-8, mgLevels=3,
              mgCycles=1, mgSmooth=None, mgCoarse=None) -> SOL:
    """Build a solver from the same keyword set the oracle's make_config takes, the way the
    reference drivers call the setters (example/TestPCG.cxx, TestKrylov.cxx, TestMG.cxx)."""
    s = ALG_CLASS[alg]()
    s.SetMaxIter(maxIter)
    s.SetMinIter(minIter)
    s.SetSavIter(savIter)
    s.SetRestart(restart)
    s.SetRelTol(relTol)
    s.SetAbsTol(absTol)
    if alg == "jacobi":
        s.SetWeight(weight)
    if alg in ("gmres", "gmres_left", "fgmres") and maxRestart:
        s.SetMaxMinRestart(maxRestart, minRestart)
    if alg == "gmres_left":
        s.SetLeftPrecond()
    if alg == "mg":
        s.cfg.mgLevels, s.cfg.mgCycles = mgLevels, mgCycles
        for name, spec in (("mgSmooth", mgSmooth), ("mgCoarse", mgCoarse)):
            if spec:
                prm = getattr(s.cfg, name + "Prm")
                for k, v in spec.items():
                    if k == "weight":
                        setattr(s.cfg, name + "Weight", v)
                    else:
                        setattr(prm, k, v)
    if pcd == "mg":
        m = MG()
        m.cfg.mgLevels, m.cfg.mgCycles = mgLevels, mgCycles
        for name, spec in (("mgSmooth", mgSmooth), ("mgCoarse", mgCoarse)):
            if spec:
                prm = getattr(m.cfg, name + "Prm")
                for k, v in spec.items():
                    if k == "weight":
                        setattr(m.cfg, name + "Weight", v)
                    else:
                        setattr(prm, k, v)
        m.SetMaxIter(pcdIter)
        m.SetMinIter(pcdIter if pcdMinIter is None else pcdMinIter)
        m.SetRelTol(pcdRelTol)
        m.SetAbsTol(pcdAbsTol)
        s.SetupPCD(m)
    if pcd == "jacobi":
        p = Jacobi(pcdWeight)
        p.SetMaxIter(pcdIter)
        p.SetMinIter(pcdIter if pcdMinIter is None else pcdMinIter)
        p.SetRelTol(pcdRelTol)
        p.SetAbsTol(pcdAbsTol)
        s.SetupPCD(p)
    return s
