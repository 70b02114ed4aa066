"""Batched Jacobi-PCG over many independent systems (fasp_gpu_batch_* in the C ABI).

``Batch`` uploads the systems as one block-diagonal CSRx matrix, picks the thread-block
shape of the persistent launch by timing the candidates on the actual batch (the
autotuner), and solves all systems and right-hand sides in one launch (FP64, or FP32 inner
iterations inside FP64 refinement).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import check, lib
from .problems import CSRMatrix, poisson2d

SHAPES = [(128, 8), (128, 16), (256, 4), (256, 8), (512, 2), (512, 4)]


def block_diagonal(mats: list[CSRMatrix]):
    """Stack CSRx matrices into one block-diagonal matrix with global column indices."""
    sys_row = np.zeros(len(mats) + 1, dtype=np.int64)
    np.cumsum([m.nrow for m in mats], out=sys_row[1:])
    nnz_off = np.zeros(len(mats) + 1, dtype=np.int64)
    np.cumsum([m.nnz for m in mats], out=nnz_off[1:])
    rp = np.empty(sys_row[-1] + 1, dtype=np.int64)
    ci = np.empty(nnz_off[-1], dtype=np.int64)
    va = np.empty(nnz_off[-1], dtype=np.float64)
    rp[-1] = nnz_off[-1]
    for k, m in enumerate(mats):
        r0, r1 = sys_row[k], sys_row[k + 1]
        rp[r0:r1] = m.rowPtr[:-1].astype(np.int64) + nnz_off[k]
        ci[nnz_off[k]:nnz_off[k + 1]] = m.colInd.astype(np.int64) + r0
        va[nnz_off[k]:nnz_off[k + 1]] = m.values
    N = int(sys_row[-1])
    return sys_row.astype(np.uint32), CSRMatrix(N, N, rp.astype(np.uint32), ci.astype(np.uint32), va)


def shifted_poisson_batch(ms, sigmas):
    """The batched workload's systems: 2D 5-point Poisson on m x m grids plus sigma I."""
    return [poisson2d(int(m), shift=float(s)) for m, s in zip(ms, sigmas)]


class _Dev:
    def __init__(self, a: np.ndarray):
        self.nbytes = a.nbytes
        self.p = C.c_void_p()
        check(lib.fasp_gpu_malloc(C.byref(self.p), max(a.nbytes, 8) + 16), "malloc")
        check(lib.fasp_gpu_memcpy_h2d(self.p, a.ctypes.data, a.nbytes), "h2d")

    def numpy(self, dtype, n):
        out = np.empty(n, dtype=dtype)
        check(lib.fasp_gpu_memcpy_d2h(out.ctypes.data, self.p, out.nbytes), "d2h")
        return out

    def __del__(self):
        if getattr(self, "p", None):
            lib.fasp_gpu_free(self.p)
            self.p = None


class Batch:
    def __init__(self, mats: list[CSRMatrix], nrhs: int, device: int = 0):
        capi.init(device)
        self.sys_row, self.A = block_diagonal(mats)
        self.count, self.nrhs, self.N = len(mats), nrhs, self.A.nrow
        self._sr = _Dev(self.sys_row)
        self._rp = _Dev(self.A.rowPtr)
        self._ci = _Dev(self.A.colInd)
        self._va = _Dev(self.A.values)
        h = C.c_void_p()
        check(lib.fasp_gpu_batch_create(self.count, self._sr.p, self.A.nnz, self._rp.p,
                                        self._ci.p, self._va.p, nrhs, C.byref(h)), "batch_create")
        self.h = h
        self.shape = (256, 4)

    def set_shape(self, block: int, per_sm: int) -> None:
        check(lib.fasp_gpu_batch_set_shape(self.h, block, per_sm), "batch_set_shape")
        self.shape = (block, per_sm)

    def solve(self, b: np.ndarray | _Dev, relTol=1e-8, maxIter=5000, precision=capi.FP64,
              innerRelTol=1e-4):
        """b: (nrhs, N) host array, or a device buffer of it. Returns (x, iters, resRel, ms)."""
        db = b if isinstance(b, _Dev) else _Dev(np.ascontiguousarray(b, dtype=np.float64))
        dx = _Dev(np.zeros(self.nrhs * self.N))
        it = np.zeros(self.count * self.nrhs, dtype=np.uint32)
        rr = np.zeros(self.count * self.nrhs, dtype=np.float64)
        check(lib.fasp_gpu_batch_solve(self.h, db.p, dx.p, relTol, maxIter, precision,
                                       innerRelTol, it.ctypes.data, rr.ctypes.data), "batch_solve")
        ms = C.c_double()
        lib.fasp_gpu_batch_last_time(self.h, C.byref(ms))
        x = dx.numpy(np.float64, self.nrhs * self.N).reshape(self.nrhs, self.N)
        return x, it.reshape(self.count, self.nrhs), rr.reshape(self.count, self.nrhs), ms.value

    def autotune(self, b, precision=capi.FP64, relTol=1e-8, reps=1):
        """Time each block shape on this batch and keep the fastest."""
        db = _Dev(np.ascontiguousarray(b, dtype=np.float64))
        best, best_ms = self.shape, float("inf")
        for shape in SHAPES:
            self.set_shape(*shape)
            t = min(self.solve(db, relTol=relTol, precision=precision)[3] for _ in range(reps))
            if t < best_ms:
                best, best_ms = shape, t
        self.set_shape(*best)
        return best, best_ms

    def __del__(self):
        if getattr(self, "h", None):
            lib.fasp_gpu_batch_destroy(self.h)
            self.h = None
