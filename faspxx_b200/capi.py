"""ctypes binding of libfasp_b200.so (include/fasp_b200.h).

Importing this module loads the in-tree CUDA library and raises ImportError when it is
missing: there is no CPU fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfasp_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is not built; run `python -m faspxx_b200.build`")

lib = C.CDLL(LIB_PATH)

# fasp_gpu_alg / precision / orth
IDENTITY, CG, BICGSTAB, GMRES, FGMRES, JACOBI, MG = 0, 1, 2, 4, 5, 11, 21
FP64, MIXED, MIXED_RELIABLE = 0, 1, 2
ORTH_CGS2, ORTH_MGS, ORTH_DCGS2 = 0, 1, 2
ERROR_CUDA, ERROR_NO_DEVICE = -101, -102


class Params(C.Structure):
    _fields_ = [("maxIter", C.c_uint32), ("minIter", C.c_uint32), ("savIter", C.c_uint32),
                ("restart", C.c_uint32), ("relTol", C.c_double), ("absTol", C.c_double)]


class Config(C.Structure):
    _fields_ = [("alg", C.c_int), ("prm", Params), ("weight", C.c_double),
                ("maxRestart", C.c_uint32), ("minRestart", C.c_uint32),
                ("pcd", C.c_int), ("pcdWeight", C.c_double), ("pcdPrm", Params),
                ("mgLevels", C.c_uint32), ("mgCycles", C.c_uint32),
                ("mgSmoothWeight", C.c_double), ("mgCoarseWeight", C.c_double),
                ("mgSmoothPrm", Params), ("mgCoarsePrm", Params),
                ("leftPrecond", C.c_int), ("precision", C.c_int), ("orth", C.c_int),
                ("innerRelTol", C.c_double), ("innerMaxIter", C.c_uint32),
                ("maxOuter", C.c_uint32), ("useGraph", C.c_int), ("persistent", C.c_int),
                ("overlapLaunch", C.c_int), ("fp32Recurrence", C.c_int)]


class Info(C.Structure):
    _fields_ = [("code", C.c_int), ("numIter", C.c_uint32), ("norm2", C.c_double),
                ("normInf", C.c_double), ("outerIter", C.c_uint32),
                ("escalations", C.c_uint32), ("launches", C.c_uint32)]


_vp, _u32, _i, _d, _sz = C.c_void_p, C.c_uint32, C.c_int, C.c_double, C.c_size_t
_P = C.POINTER

SIGNATURES = {
    "fasp_gpu_init": (_i, [_i]),
    "fasp_gpu_abi_version": (_i, []),
    "fasp_gpu_strerror": (C.c_char_p, [_i]),
    "fasp_gpu_default_config": (None, [_P(Config), _i]),
    "fasp_gpu_malloc": (_i, [_P(_vp), _sz]),
    "fasp_gpu_free": (_i, [_vp]),
    "fasp_gpu_memcpy_h2d": (_i, [_vp, _vp, _sz]),
    "fasp_gpu_memcpy_d2h": (_i, [_vp, _vp, _sz]),
    "fasp_gpu_memset": (_i, [_vp, _i, _sz]),
    "fasp_gpu_synchronize": (_i, []),
    "fasp_gpu_host_alloc": (_i, [_P(_vp), _sz]),
    "fasp_gpu_host_free": (_i, [_vp]),
    "fasp_gpu_mat_create": (_i, [_u32, _u32, _u32, _vp, _vp, _vp, _P(_vp)]),
    "fasp_gpu_mat_create_device": (_i, [_u32, _u32, _u32, _vp, _vp, _vp, _P(_vp)]),
    "fasp_gpu_mat_create_coo": (_i, [_u32, _u32, _u32, _vp, _vp, _vp, _i, _P(_vp)]),
    "fasp_gpu_mat_create_csr_raw": (_i, [_u32, _u32, _u32, _vp, _vp, _vp, _i, _P(_vp)]),
    "fasp_gpu_mat_create_stencil": (_i, [_u32, _u32, _u32, _u32, _vp, _vp, _vp, _vp, _P(_vp)]),
    "fasp_gpu_mat_mult": (_i, [_vp, _vp, _P(_vp)]),
    "fasp_gpu_mat_add": (_i, [C.c_double, _vp, C.c_double, _vp, _P(_vp)]),
    "fasp_gpu_mat_destroy": (_i, [_vp]),
    "fasp_gpu_mat_info": (_i, [_vp, _P(_u32), _P(_u32), _P(_u32)]),
    "fasp_gpu_mat_download": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "fasp_gpu_mat_apply": (_i, [_vp, _vp, _vp]),
    "fasp_gpu_mat_residual": (_i, [_vp, _vp, _vp, _vp]),
    "fasp_gpu_mat_transpose": (_i, [_vp, _P(_vp)]),
    "fasp_gpu_mat_diag": (_i, [_vp, _vp]),
    "fasp_gpu_mat_autotune": (_i, [_vp, _P(_i)]),
    "fasp_gpu_mat_set_lanes": (_i, [_vp, _i]),
    "fasp_gpu_mat_set_rowclass": (_i, [_vp, _i]),
    "fasp_gpu_mat_rowclass_info": (_i, [_vp, _P(_i), _P(_u32), _P(_u32), _P(_u32)]),
    "fasp_gpu_mat_time_apply": (_i, [_vp, _u32, _i, _i, _P(_d)]),
    "fasp_gpu_mat_set_col16": (_i, [_vp, _i]),
    "fasp_gpu_mat_col16_info": (_i, [_vp, _P(_i), _P(_i)]),
    "fasp_gpu_mat_tile_info": (_i, [_vp, _P(_u32), _P(_i), _P(_i), _P(_i)]),
    "fasp_gpu_tile_timeouts": (_i, [_P(_u32)]),
    "fasp_gpu_mat_sampled_outer": (_i, [_vp, _vp, _vp, _d, _vp]),
    "fasp_gpu_mat_mult_transpose_add": (_i, [_vp, _vp, _vp, _vp]),
    "fasp_gpu_mat_apply_async": (_i, [_vp, _vp, _vp, _vp]),
    "fasp_gpu_mat_residual_async": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "fasp_gpu_mat_mult_transpose_add_async": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "fasp_gpu_mat_sampled_outer_async": (_i, [_vp, _vp, _vp, _d, _vp, _vp]),
    "fasp_gpu_vec_dot": (_i, [_u32, _vp, _vp, _P(_d)]),
    "fasp_gpu_vec_norm2": (_i, [_u32, _vp, _P(_d)]),
    "fasp_gpu_vec_norminf": (_i, [_u32, _vp, _P(_d)]),
    "fasp_gpu_vec_axpy": (_i, [_u32, _d, _vp, _vp]),
    "fasp_gpu_vec_xpay": (_i, [_u32, _d, _vp, _vp]),
    "fasp_gpu_vec_axpby": (_i, [_u32, _d, _d, _vp, _vp]),
    "fasp_gpu_vec_waxpby": (_i, [_u32, _d, _vp, _d, _vp, _vp]),
    "fasp_gpu_vec_scale": (_i, [_u32, _d, _vp]),
    "fasp_gpu_vec_dot_noalloc": (_i, [_u32, _vp, _vp, _P(_d)]),
    "fasp_gpu_vec_dot_async": (_i, [_u32, _vp, _vp, _vp, _vp]),
    "fasp_gpu_vec_norm2_async": (_i, [_u32, _vp, _vp, _vp]),
    "fasp_gpu_vec_norminf_async": (_i, [_u32, _vp, _vp, _vp]),
    "fasp_gpu_vec_axpy_async": (_i, [_u32, _d, _vp, _vp, _vp]),
    "fasp_gpu_vec_xpay_async": (_i, [_u32, _d, _vp, _vp, _vp]),
    "fasp_gpu_vec_axpby_async": (_i, [_u32, _d, _d, _vp, _vp, _vp]),
    "fasp_gpu_vec_waxpby_async": (_i, [_u32, _d, _vp, _d, _vp, _vp, _vp]),
    "fasp_gpu_vec_scale_async": (_i, [_u32, _d, _vp, _vp]),
    "fasp_gpu_solver_create": (_i, [_P(Config), _P(_vp)]),
    "fasp_gpu_solver_setup": (_i, [_vp, _vp]),
    "fasp_gpu_solver_set_mg_transfer": (_i, [_vp, _u32, _vp, _vp, _vp]),
    "fasp_gpu_solver_solve": (_i, [_vp, _vp, _vp, _P(Info)]),
    "fasp_gpu_solver_solve_host": (_i, [_vp, _vp, _vp, _P(Info)]),
    "fasp_gpu_solver_solve_async": (_i, [_vp, _vp, _vp, _P(Info), _vp]),
    "fasp_gpu_solver_history": (_i, [_vp, _vp, _u32, _P(_u32)]),
    "fasp_gpu_solver_clean": (_i, [_vp]),
    "fasp_gpu_solver_destroy": (_i, [_vp]),
    "fasp_gpu_solver_last_time": (_i, [_vp, _P(_d)]),
    "fasp_gpu_solver_kernel_times": (_i, [_vp, _u32, _i, _P(_d)]),
    "fasp_gpu_solver_set_barrier_limit": (_i, [_vp, _u32]),
    "fasp_gpu_solver_solve_adjoint": (_i, [_vp, _vp, _vp, _P(Info)]),
    "fasp_gpu_solver_solve_adjoint_async": (_i, [_vp, _vp, _vp, _P(Info), _vp]),
    "fasp_gpu_batch_create": (_i, [_u32, _vp, _u32, _vp, _vp, _vp, _u32, _P(_vp)]),
    "fasp_gpu_batch_set_shape": (_i, [_vp, _i, _i]),
    "fasp_gpu_batch_solve": (_i, [_vp, _vp, _vp, _d, _u32, _i, _d, _vp, _vp]),
    "fasp_gpu_batch_solve_async": (_i, [_vp, _vp, _vp, _d, _u32, _i, _d, _vp, _vp, _vp]),
    "fasp_gpu_batch_last_time": (_i, [_vp, _P(_d)]),
    "fasp_gpu_batch_destroy": (_i, [_vp]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(lib, _name)  # AttributeError = a declared entry point is missing
    _f.restype = _res
    _f.argtypes = _args


class FaspError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib.fasp_gpu_strerror(code).decode()
        super().__init__(f"{where}: {msg} ({code})")
        self.code = code


def check(code: int, where: str) -> int:
    if code != 0:
        raise FaspError(code, where)
    return code


def default_config(alg: int) -> Config:
    cfg = Config()
    lib.fasp_gpu_default_config(C.byref(cfg), alg)
    return cfg


_initialised = {}


def init(device: int = 0) -> None:
    if _initialised.get(device):
        return
    check(lib.fasp_gpu_init(device), "fasp_gpu_init")
    _initialised[device] = True
