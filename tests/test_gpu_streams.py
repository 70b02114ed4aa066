"""Stream-ordered entry points (the _async forms in include/fasp_b200.h).

A caller's stream runs slow work and then the kernel that writes the right-hand side; the
library call is issued right after, on the same stream, with no synchronisation. The call
must see the written input (it is ordered after the caller's earlier work) and the
caller's next kernel on the stream must see its output (ordered after the call). Without
the ordering the library's own stream would start at once and read a zero right-hand
side. The caller's stream and kernels come from PyTorch (test plumbing only).

Bars: the solve equals the blocking solve bit for bit (same iterations, same x); Apply,
MultTransposeAdd and the dot product equal their blocking forms bit for bit; the AXPY
equals y + a x to 1e-15 relative (one fused multiply-add per entry).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    from faspxx_b200 import capi, problems as P, sol
    capi.init(0)
    torch.cuda.init()
    return torch, capi, P, sol


def _busy(torch, s, reps=8):
    """Queue slow work on stream s: chained FP32 products of 8192^2 matrices (about 10 ms
    each), so that anything not ordered after it would run first."""
    with torch.cuda.stream(s):
        a = torch.randn(8192, 8192, device="cuda")
        for _ in range(reps):
            a = torch.tanh(a @ a * 1e-4)
    return a


def test_solve_async_ordered_on_caller_stream(env):
    torch, capi, P, sol = env
    A = P.poisson3d(48)
    b = A.matvec(P.seeded_uniform(A.nrow, 42))
    M = sol.MAT(A)
    s = sol.configure("cg", maxIter=1000, relTol=1e-8, absTol=0.0, pcd="jacobi", pcdIter=1)
    s.Setup(M)
    x_ref = np.zeros(A.nrow)
    assert s.Solve(b, x_ref) == 0
    it_ref = s.GetIterations()

    st = torch.cuda.Stream()
    src = torch.tensor(b, device="cuda")
    bt = torch.zeros(A.nrow, dtype=torch.float64, device="cuda")
    xt = torch.zeros(A.nrow, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _busy(torch, st)
    with torch.cuda.stream(st):
        bt.copy_(src)                      # the caller's kernel that forms b
    info = capi.Info()
    code = capi.lib.fasp_gpu_solver_solve_async(s.h, C.c_void_p(bt.data_ptr()),
                                                C.c_void_p(xt.data_ptr()), C.byref(info),
                                                C.c_void_p(st.cuda_stream))
    assert code == 0 and info.code == 0
    with torch.cuda.stream(st):
        out = xt.clone()                   # the caller's next kernel reads x
    st.synchronize()
    assert info.numIter == it_ref
    assert np.array_equal(out.cpu().numpy(), x_ref)


def test_operator_and_vec_async(env):
    torch, capi, P, sol = env
    lib = capi.lib
    A = P.convdiff3d(24, 10.0)
    M = sol.MAT(A)
    rng = np.random.default_rng(4)
    v, v2 = rng.standard_normal(A.nrow), rng.standard_normal(A.nrow)
    w_ref, t_ref = sol.DVec(A.nrow), sol.DVec(A.nrow)
    M.Apply(sol.DVec.from_numpy(v), w_ref)
    M.MultTransposeAdd(sol.DVec.from_numpy(v), sol.DVec.from_numpy(v2), t_ref)
    dot_ref = sol.DVec.from_numpy(v).Dot(sol.DVec.from_numpy(v2))

    st = torch.cuda.Stream()
    src, src2 = torch.tensor(v, device="cuda"), torch.tensor(v2, device="cuda")
    vt = torch.zeros_like(src)
    v2t = torch.zeros_like(src)
    wt, tt = torch.zeros_like(src), torch.zeros_like(src)
    dres = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _busy(torch, st)
    with torch.cuda.stream(st):
        vt.copy_(src)
        v2t.copy_(src2)
    hs = C.c_void_p(st.cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    assert lib.fasp_gpu_mat_apply_async(M.h, p(vt), p(wt), hs) == 0
    assert lib.fasp_gpu_mat_mult_transpose_add_async(M.h, p(vt), p(v2t), p(tt), hs) == 0
    assert lib.fasp_gpu_vec_dot_async(A.nrow, p(vt), p(v2t), p(dres), hs) == 0
    # AXPY after the dot on the same caller stream: y = v2 + 0.5 v
    assert lib.fasp_gpu_vec_axpy_async(A.nrow, 0.5, p(vt), p(v2t), hs) == 0
    with torch.cuda.stream(st):
        outs = [wt.clone(), tt.clone(), dres.clone(), v2t.clone()]
    st.synchronize()
    w, t, d, y = (o.cpu().numpy() for o in outs)
    assert np.array_equal(w, w_ref.numpy())
    assert np.array_equal(t, t_ref.numpy())
    assert d[0] == dot_ref
    assert np.allclose(y, v2 + 0.5 * v, rtol=1e-15, atol=1e-15)
