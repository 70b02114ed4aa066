"""fasp_gpu_vec_dot_noalloc: the dot product for callers that cannot allocate device memory
(an application whose memory pool owns the device memory, or a latency-critical loop where
cudaMalloc/cudaFree would synchronize). It keeps its reduction scratch in a static device
array instead of allocating; this test checks it through the C ABI against
fasp_gpu_vec_dot, the allocating entry point, on two calls in a row (the array keeps the
previous call's contents), from a fresh host thread that never selected a device (the
entry point runs on the library's device), and checks that sizes beyond the array's limit
are refused. The test allocates its own inputs; the entry point does not.

This file is named to be collected last, and passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative, as for the other VEC reductions
MAX_N = 8_388_608


def _dev(capi, host):
    p = C.c_void_p()
    capi.check(capi.lib.fasp_gpu_malloc(C.byref(p), host.nbytes + 16), "malloc")
    capi.check(capi.lib.fasp_gpu_memcpy_h2d(p, host.ctypes.data, host.nbytes), "h2d")
    return p


def test_noalloc_dot_matches_allocating_dot_twice():
    from faspxx_b200 import capi
    capi.init(0)
    lib = capi.lib
    rng = np.random.default_rng(17)
    bufs = []
    try:
        for n in (2_097_152, 2_097_152, 1_000_003, 5, MAX_N):
            a, b = rng.standard_normal(n), rng.standard_normal(n)
            da, db = _dev(capi, a), _dev(capi, b)
            bufs += [da, db]
            got = []
            for _ in range(2):  # two calls in a row share the static scratch
                r = C.c_double(np.nan)
                capi.check(lib.fasp_gpu_vec_dot_noalloc(n, da, db, C.byref(r)), "noalloc")
                got.append(r.value)
            ref = C.c_double()
            capi.check(lib.fasp_gpu_vec_dot(n, da, db, C.byref(ref)), "dot")
            scale = float(np.abs(a * b).sum())
            for g in got:
                assert abs(g - ref.value) <= TOL * scale, (n, g, ref.value)
            assert got[0] == got[1]  # fixed reduction order: the same bits every call
            assert abs(got[0] - float(a @ b)) <= 1e-12 * scale
            lib.fasp_gpu_free(da)
            lib.fasp_gpu_free(db)
            bufs.clear()
    finally:
        for p in bufs:
            lib.fasp_gpu_free(p)


def test_noalloc_dot_from_a_fresh_thread():
    """A worker thread with no CUDA device selected gets the library's device."""
    import threading
    from faspxx_b200 import capi
    capi.init(0)
    lib = capi.lib
    rng = np.random.default_rng(23)
    n = 1_048_579
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    da, db = _dev(capi, a), _dev(capi, b)
    try:
        ref = C.c_double()
        capi.check(lib.fasp_gpu_vec_dot(n, da, db, C.byref(ref)), "dot")
        out = {}

        def worker():
            r = C.c_double(np.nan)
            out["codes"] = [lib.fasp_gpu_vec_dot_noalloc(n, da, db, C.byref(r))]
            out["vals"] = [r.value]
            out["codes"].append(lib.fasp_gpu_vec_dot_noalloc(n, da, db, C.byref(r)))
            out["vals"].append(r.value)

        t = threading.Thread(target=worker)
        t.start()
        t.join()
        assert out["codes"] == [0, 0]
        scale = float(np.abs(a * b).sum())
        for g in out["vals"]:
            assert abs(g - ref.value) <= TOL * scale, (g, ref.value)
    finally:
        lib.fasp_gpu_free(da)
        lib.fasp_gpu_free(db)


def test_noalloc_dot_rejects_sizes_beyond_its_scratch():
    from faspxx_b200 import capi
    capi.init(0)
    r = C.c_double(1.0)
    # refused before any device access: the pointers are never read
    code = capi.lib.fasp_gpu_vec_dot_noalloc(MAX_N + 1, C.c_void_p(16), C.c_void_p(16),
                                            C.byref(r))
    assert code == -14
    assert r.value == 1.0
    assert capi.lib.fasp_gpu_vec_dot_noalloc(0, None, None, C.byref(r)) == 0 and r.value == 0.0
