"""Differentiable sparse solve x = A^-1 b as a torch.autograd.Function (a test harness over
the C ABI; the library itself has no PyTorch dependency).

Forward: CG (FP64, or FP32-inner mixed precision) on the CSRx matrix with the given values.
Backward, for an upstream gradient g = dL/dx:
    lambda = A^-T g           adjoint solve, the same Krylov kernels on the exact CSC
                              transpose (MAT::TransInPlace order), built once and cached
    dL/db  = lambda
    dL/dA_k = -lambda[row(k)] * x[col(k)]   sampled outer product on A's sparsity pattern
The forward x is saved, not recomputed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi
from .capi import check, lib


class SparseSystem:
    """Fixed sparsity structure (rowPtr, colInd) with solver settings; values vary."""

    def __init__(self, rowPtr: np.ndarray, colInd: np.ndarray, n: int, relTol: float = 1e-10,
                 maxIter: int = 20000, precision: int = capi.FP64, pcd_weight: float = 1.0,
                 device: int = 0):
        capi.init(device)
        self.n = int(n)
        self.nnz = int(colInd.shape[0])
        self.rowPtr = torch.as_tensor(np.ascontiguousarray(rowPtr, np.uint32).view(np.int32),
                                      device=f"cuda:{device}")
        self.colInd = torch.as_tensor(np.ascontiguousarray(colInd, np.uint32).view(np.int32),
                                      device=f"cuda:{device}")
        self.relTol, self.maxIter, self.precision = relTol, maxIter, precision
        self.pcd_weight = pcd_weight
        self._mat = None
        self._solver = None
        self._values_version = None
        self._values_ref = None

    def _bind(self, values: torch.Tensor):
        # the tensor object itself is held, so its storage cannot be recycled under the key
        key = (id(values), values._version)
        if self._mat is not None and self._values_version == key and \
                self._values_ref is values:
            return
        self._values_ref = values
        self.close()
        torch.cuda.synchronize()
        m = C.c_void_p()
        check(lib.fasp_gpu_mat_create_device(self.n, self.n, self.nnz, self.rowPtr.data_ptr(),
                                             self.colInd.data_ptr(), values.data_ptr(),
                                             C.byref(m)), "mat_create_device")
        self._mat = m
        cfg = capi.default_config(capi.CG)
        cfg.prm.maxIter, cfg.prm.minIter = self.maxIter, 0
        cfg.prm.relTol, cfg.prm.absTol = self.relTol, 0.0
        cfg.pcd, cfg.pcdWeight = 1, self.pcd_weight
        cfg.pcdPrm.maxIter = cfg.pcdPrm.minIter = 1
        cfg.precision = self.precision
        s = C.c_void_p()
        check(lib.fasp_gpu_solver_create(C.byref(cfg), C.byref(s)), "solver_create")
        check(lib.fasp_gpu_solver_setup(s, m), "solver_setup")
        self._solver = s
        self._values_version = key

    def solve(self, values: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        self._bind(values)
        x = torch.zeros_like(b)
        info = capi.Info()
        torch.cuda.synchronize()
        check(lib.fasp_gpu_solver_solve(self._solver, b.data_ptr(), x.data_ptr(),
                                        C.byref(info)), "solve")
        if info.code != 0:
            raise capi.FaspError(info.code, "forward solve")
        return x

    def adjoint(self, values: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
        self._bind(values)
        lam = torch.zeros_like(g)
        info = capi.Info()
        torch.cuda.synchronize()
        check(lib.fasp_gpu_solver_solve_adjoint(self._solver, g.data_ptr(), lam.data_ptr(),
                                                C.byref(info)), "adjoint")
        if info.code != 0:
            raise capi.FaspError(info.code, "adjoint solve")
        return lam

    def outer(self, values, lam: torch.Tensor, x: torch.Tensor, scale: float) -> torch.Tensor:
        self._bind(values)
        out = torch.empty(self.nnz, dtype=torch.float64, device=lam.device)
        torch.cuda.synchronize()
        check(lib.fasp_gpu_mat_sampled_outer(self._mat, lam.data_ptr(), x.data_ptr(), scale,
                                             out.data_ptr()), "sampled_outer")
        return out

    def close(self):
        if self._solver is not None:
            lib.fasp_gpu_solver_destroy(self._solver)
            self._solver = None
        if self._mat is not None:
            lib.fasp_gpu_mat_destroy(self._mat)
            self._mat = None

    def __del__(self):
        self.close()


class SparseSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values: torch.Tensor, b: torch.Tensor, system: SparseSystem):
        values = values.detach().contiguous()
        b = b.detach().contiguous()
        x = system.solve(values, b)
        ctx.system = system
        ctx.save_for_backward(values, x)
        return x

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        values, x = ctx.saved_tensors
        system = ctx.system
        lam = system.adjoint(values, g.detach().contiguous())
        dA = system.outer(values, lam, x, -1.0) if ctx.needs_input_grad[0] else None
        db = lam if ctx.needs_input_grad[1] else None
        return dA, db, None


def sparse_solve(values: torch.Tensor, b: torch.Tensor, system: SparseSystem) -> torch.Tensor:
    return SparseSolve.apply(values, b, system)
