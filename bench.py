#!/usr/bin/env python
"""Benchmark: time to an FP64 relative residual of 1e-8 on the 3D 7-point Poisson problem
(128^3 grid, n = 2,097,152, nnz = 14,581,760), Jacobi-preconditioned CG (weight 1, one
sweep), mixed precision (FP32 CG iterations with FP64 reliable updates of x and r) against
plain FP64 CG on the same B200, plus SpMV GB/s. One JSON line on rank 0. The restarted
variant (FP32 inner CG solves inside FP64 iterative refinement) is timed beside them.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one complete solve from x0 = 0 of A x = b, b = A x*, x* ~ U[0,1) (seed 42).
`value` is the device time of the mixed-precision solve (CUDA events on the solver's
stream, inputs resident in HBM); `e2e` the same solve through the host entry point with
b and x0 copied in from pinned host memory and x copied back every step. Under torchrun
every rank solves its own replica of the system (the single system does not shard) and
the slowest rank's time is reported. `--impl reference` times the FASP++ reference
(compiled from its own sources into oracle/_ref) on the host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 128
METRIC = ("Time-to-1e-8 FP64 residual, 128³ Poisson CG: mixed vs FP64 on B200; "
          "SpMV GB/s")
REL_TOL = 1e-8
MAX_ITER = 3000


def problem(ngrid: int):
    from faspxx_b200 import problems as P
    A = P.poisson3d(ngrid)
    xs = P.seeded_uniform(A.nrow, 42)
    b = A.matvec(xs)
    return A, b


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(key: str):
    """DRAM bytes (read + write) per launch of a kernel at this workload from the committed
    ncu summaries (profiles/*.txt lines "dram_bytes_per_launch <key> <bytes>", key = kernel
    and matrix form); null when no capture of the current kernel exists."""
    prefix = key
    try:
        for fn in sorted(os.listdir(os.path.join(ROOT, "profiles"))):
            if not fn.endswith(".txt"):
                continue
            for line in open(os.path.join(ROOT, "profiles", fn)):
                f = line.split()
                if len(f) == 3 and f[0] == "dram_bytes_per_launch" and f[1] == prefix:
                    return int(float(f[2]))
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a timed region.

    nvidia-smi's start-up (NVML initialisation, device attach) disturbs GPU work that runs
    at the same moment, so __enter__ waits for its first sample before the timed region
    starts; samples from before the region are dropped when later ones exist."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.rows = []
        self.first = 0

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        t0 = time.perf_counter()
        while not self.rows and time.perf_counter() - t0 < 5.0:
            time.sleep(0.01)
        time.sleep(0.05)
        self.first = len(self.rows)
        return self

    def __exit__(self, *exc):
        if self.proc is None:
            return False
        time.sleep(0.25)  # at least one sample ends inside or right after the region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=5)
        return False

    def summary(self):
        rows = self.rows[self.first:] or self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        self.rows = rows
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit())
        loaded = [s for s in sm if s > 0.5 * smax] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(self.rows)}


def l2_copy_gbs(device: int) -> float:
    """Measured L2-resident copy bandwidth on this GPU: torch copy_ between two 24 MB
    buffers (48 MB of the 126 MB L2), 64 copies captured in one CUDA graph and replayed,
    CUDA events; bytes read + written per copy over the mean copy time (launch gaps
    included, as in the solver's graphs)."""
    import torch
    dev = torch.device("cuda", device)
    n = 6 << 20
    a = torch.ones(n, device=dev)
    b = torch.empty_like(a)
    s = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(s):
        for _ in range(4):
            b.copy_(a)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            for _ in range(64):
                b.copy_(a)
        g.replay()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        best = float("inf")
        for _ in range(5):
            e0.record(s)
            g.replay()
            e1.record(s)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 64)
    del g
    return 2 * 4 * n / (best * 1e-3) / 1e9


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return dist


def dist_max(dist, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---- CPU reference / baseline ---------------------------------------------------------

def reference_sample(A, b, sample_iters: int, kind: str = "ref"):
    """Time `sample_iters` Jacobi-PCG iterations of the CPU oracle (the reference compiled
    from its own sources when kind == 'ref') from x0 = 0; returns ms per iteration."""
    from oracle import oracle as O
    kw = dict(maxIter=sample_iters, minIter=0, relTol=1e-300, absTol=0.0, pcd="jacobi",
              pcdWeight=1.0, pcdIter=1)
    s = O.Solver(kind, A, "cg", **kw)
    x0 = np.zeros(A.nrow)
    t = time.perf_counter()
    r = s.solve(b, x0)
    dt = time.perf_counter() - t
    return dt * 1e3 / max(1, r.iters), r.iters


def reference_full(A, b, kind: str = "ref"):
    from oracle import oracle as O
    s = O.Solver(kind, A, "cg", maxIter=MAX_ITER, minIter=0, relTol=REL_TOL, absTol=0.0,
                 pcd="jacobi", pcdWeight=1.0, pcdIter=1)
    t = time.perf_counter()
    r = s.solve(b, np.zeros(A.nrow))
    return (time.perf_counter() - t) * 1e3, r.iters, r.code


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import oracle as O
    kind = "ref" if os.path.exists(O.REF_SO) else "port"
    A, b = problem(args.size)
    # warm-up steps: short samples (20 iterations each); timed steps: complete solves
    for _ in range(args.warmup):
        reference_sample(A, b, 20, kind)
    full, iters, code = [], 0, 0
    for _ in range(args.steps):
        ms, iters, code = reference_full(A, b, kind)
        full.append(ms)
    value = statistics.mean(full)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(value, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3D Poisson 7-point {args.size}^3, Jacobi-PCG, rtol 1e-8",
                   "n": A.nrow, "nnz": A.nnz, "solver": "FASP++ CG + Jacobi(w=1, 1 sweep)"},
        "cpu_baseline": {"value": round(value, 3), "unit": "ms", "cores": 1,
                         "kind": "reference" if kind == "ref" else "port",
                         "sample": f"each timed step is one complete solve from x0 = 0 to "
                                   f"rtol 1e-8 ({iters} iterations, code {code}); warm-up "
                                   f"steps are 20-iteration samples; the reference's solve "
                                   f"path is serial (its OpenMP pragmas are off by default "
                                   f"and gave no speed-up), so one core"},
        "e2e": {"value": round(value, 3), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "full_solve_ms": [round(t, 1) for t in full], "iterations": iters,
    }
    print(json.dumps(line))
    return 0


# ---- GPU arm ------------------------------------------------------------------------

def run_ours(args):
    ws, rank, local = dist_env()
    dist = dist_init(ws)
    from faspxx_b200 import capi, sol
    capi.init(local)
    lib = capi.lib
    A, b = problem(args.size)
    n, nnz = A.nrow, A.nnz
    M = sol.MAT(A)
    lanes = M.Autotune() if not args.lanes else (M.SetLanes(args.lanes) or args.lanes)
    if args.form == "csr":
        M.SetRowClass(0)
    if args.profile_apply:
        # for ncu: MAT::Apply on FP64 in the chosen form, 3 warm-up and 4 timed launches
        sp = C.c_double()
        capi.check(lib.fasp_gpu_mat_time_apply(M.h, 4, 0, 0, C.byref(sp)), "time_apply")
        print(f"profile-apply form {M.RowClassInfo()[0]} tiles {M.TileInfo()} "
              f"{sp.value * 1e3:.1f} us per launch")
        return 0

    def make(precision):
        s = sol.CG()
        s.SetMaxIter(MAX_ITER)
        s.SetMinIter(0)
        s.SetRelTol(REL_TOL)
        s.SetAbsTol(0.0)
        p = sol.Jacobi(1.0)
        p.SetMaxIter(1)
        p.SetMinIter(1)
        s.SetupPCD(p)
        if precision == capi.MIXED:
            s.SetPrecision(capi.MIXED, innerRelTol=args.inner_tol, maxOuter=50)
        elif precision == capi.MIXED_RELIABLE:
            s.SetPrecision(capi.MIXED_RELIABLE, innerRelTol=args.delta)
        s.Setup(M)
        return s

    mixed, fp64 = make(capi.MIXED_RELIABLE), make(capi.FP64)
    if args.profile_solve:
        # for a time-only ncu launch list: three identical mixed solves and nothing else
        db, dx = sol.DVec.from_numpy(b), sol.DVec(n)
        for _ in range(3):
            dx.Zero()
            code = mixed.Solve(db, dx)
            print(f"profile-solve code {code} iterations {mixed.GetIterations()} "
                  f"{mixed.LastTimeMs():.3f} ms launches {mixed.info.launches}")
        return 0
    restarted = make(capi.MIXED)
    if args.profile:
        # 3 warm-up + 1 launch of cg_spmv and cg_update per engine: FP32 first, then FP64
        km = (C.c_double * 3)()
        for s in (mixed, fp64):
            capi.check(lib.fasp_gpu_solver_kernel_times(s.h, 1, 0, km), "kernel_times")
            print(f"profile lanes={lanes} spmv {km[0]*1e3:.1f} us update {km[1]*1e3:.1f} us "
                  f"persistent iteration {km[2]*1e3:.1f} us")
        return 0
    db = sol.DVec.from_numpy(b)
    dx = sol.DVec(n)
    # 256 MB, read between solves (a norm: no stores) to evict L2 (126 MB) and leave it
    # holding clean lines, so no write-back of dirty lines lands in the timed solve
    l2flush = sol.DVec(32 << 20)

    def solve(s):
        dx.Zero()  # x0 = 0 on the device
        l2flush.Norm2()
        code = s.Solve(db, dx)
        if code != 0:
            raise RuntimeError(f"solve failed with code {code}")
        return s.LastTimeMs(), s.info.numIter, s.info.launches, s.info.outerIter

    for _ in range(args.warmup):
        solve(mixed)
        solve(fp64)
        solve(restarted)

    # accuracy of each variant: FP64 residual and error against an FP64 CG solve to 1e-13
    tight = make(capi.FP64)
    tight.SetRelTol(1e-13)
    dx.Zero()
    tight.Solve(db, dx)
    xref = dx.numpy()
    del tight

    def accuracy(s):
        solve(s)
        x = dx.numpy()
        r = b - A.matvec(x)
        return (float(np.linalg.norm(r) / np.linalg.norm(b)),
                float(np.linalg.norm(x - xref) / np.linalg.norm(xref)))

    acc_mixed, acc_fp64 = accuracy(mixed), accuracy(fp64)

    lib.fasp_gpu_synchronize()
    barrier(dist)
    with ClockSampler(local) as clk:
        times, its, launches, outer = [], [], 0, 0
        for _ in range(args.steps):
            t, it, la, ou = solve(mixed)
            times.append(t)
            its.append(it)
            launches += la + 1
            outer = ou
        lib.fasp_gpu_synchronize()
        times64, its64 = [], []
        for _ in range(args.steps):
            t, it, la, _ = solve(fp64)
            times64.append(t)
            its64.append(it)
        lib.fasp_gpu_synchronize()
        timesR, itsR, outerR = [], [], 0
        for _ in range(args.steps):
            t, it, la, outerR = solve(restarted)
            timesR.append(t)
            itsR.append(it)
        lib.fasp_gpu_synchronize()
    barrier(dist)
    clocks = clk.summary()
    mixed_ms = dist_max(dist, statistics.mean(times))
    fp64_ms = dist_max(dist, statistics.mean(times64))
    restarted_ms = dist_max(dist, statistics.mean(timesR))

    # the same solves with the matrix in plain CSR form: what a general FASP++ matrix (no
    # row-class or stencil-mask compression) gets
    rc_mode_used = M.RowClassInfo()[0]
    M.SetRowClass(0)
    csr_res = {}
    for col16 in (False, True):
        M.SetCol16(col16)
        for tag, prec in (("mixed", capi.MIXED_RELIABLE), ("fp64", capi.FP64)):
            sc = make(prec)
            for _ in range(2):
                solve(sc)
            ts = [solve(sc) for _ in range(args.steps)]
            csr_res[(tag, col16)] = (dist_max(dist, statistics.mean(t[0] for t in ts)),
                                     ts[-1][1])
            del sc
    M.SetCol16(False)
    M.SetRowClass(rc_mode_used)

    # end to end: host b, x0 in pinned memory -> device -> solve -> x back to host
    hb = C.c_void_p()
    hx = C.c_void_p()
    capi.check(lib.fasp_gpu_host_alloc(C.byref(hb), n * 8), "host_alloc")
    capi.check(lib.fasp_gpu_host_alloc(C.byref(hx), n * 8), "host_alloc")
    bh = np.ctypeslib.as_array((C.c_double * n).from_address(hb.value))
    xh = np.ctypeslib.as_array((C.c_double * n).from_address(hx.value))
    bh[:] = b
    e2e = []
    for i in range(args.warmup + args.steps):
        xh[:] = 0.0
        lib.fasp_gpu_synchronize()
        t0 = time.perf_counter()
        code = lib.fasp_gpu_solver_solve_host(mixed.h, hb, hx, C.byref(mixed.info))
        t1 = time.perf_counter()
        if code != 0 or mixed.info.code != 0:
            raise RuntimeError("end-to-end solve failed")
        if i >= args.warmup:
            e2e.append((t1 - t0) * 1e3)
    e2e_ms = dist_max(dist, statistics.mean(e2e))
    e2e_err = float(np.linalg.norm(xh - xref) / np.linalg.norm(xref))
    lib.fasp_gpu_host_free(hb)
    lib.fasp_gpu_host_free(hx)

    # kernel rooflines (each kernel alone, CUDA events on the library's stream)
    hbm, peak_kind = peaks()
    km = (C.c_double * 3)()
    capi.check(lib.fasp_gpu_solver_kernel_times(mixed.h, 30, 1, km), "kernel_times")
    k64 = (C.c_double * 3)()
    capi.check(lib.fasp_gpu_solver_kernel_times(fp64.h, 30, 1, k64), "kernel_times")
    # the same kernels as they run inside the solve: back to back on the solver's own data
    kwarm = (C.c_double * 3)()
    capi.check(lib.fasp_gpu_solver_kernel_times(mixed.h, 200, 0, kwarm), "kernel_times")
    try:
        l2_gbs = l2_copy_gbs(local)
    except Exception:  # torch missing: the L2 fraction is left out
        l2_gbs = None
    sp = C.c_double()
    capi.check(lib.fasp_gpu_mat_time_apply(M.h, 30, 0, 1, C.byref(sp)), "time_apply")
    rc_mode, rc_classes, rc_entries, rc_stencil = M.RowClassInfo()
    rc_on = rc_mode > 0
    sp_csr = C.c_double()
    sp_csr_seq = C.c_double()
    M.SetRowClass(0)
    capi.check(lib.fasp_gpu_mat_time_apply(M.h, 30, 0, 1, C.byref(sp_csr)), "time_apply")
    # the CSR inputs (217 MB at 128^3) exceed L2: back-to-back launches stream from HBM
    capi.check(lib.fasp_gpu_mat_time_apply(M.h, 50, 0, 0, C.byref(sp_csr_seq)), "time_apply")
    M.SetRowClass(rc_mode)
    # algorithmic bytes per launch (compulsory traffic); the matrix streams either the CSR
    # arrays (values + column indices + row pointers) or one 2-byte class id / stencil mask
    # per row (the class table stays in L1/L2, the stencil travels as kernel parameters)
    mat32 = 2 * n if rc_on else 8 * nnz + 4 * (n + 1)
    mat64 = 2 * n if rc_on else 12 * nnz + 4 * (n + 1)
    # FP32 iterations on this matrix (one Jacobi diagonal value) run the one-reduction
    # engine: cg_spmv reads r (gathered), p, q, x and writes p, q, x (x += alpha p of the
    # last iteration); cg_update_r reads r, q and writes r
    b_spmv32 = mat32 + 4 * n * 7
    b_upd32 = 4 * n * 3
    b_spmv64 = mat64 + 8 * n * 4
    b_upd64 = 8 * n * 5 + 8 * n * 3
    b_apply = mat64 + 16 * n
    b_apply_csr = 12 * nnz + 4 * (n + 1) + 16 * n
    gbs = lambda byt, ms: byt / (ms * 1e-3) / 1e9  # noqa: E731
    if km[2] > 0:
        # the persistent kernel runs the whole FP32 inner solve: one iteration = both phases
        b_it32 = b_spmv32 + b_upd32
        ach = gbs(b_it32, km[2])
        roofline = {"kernel": "cg_persistent<float,JAC> (one FP32 PCG iteration: SpMV + p "
                              "update + x,r,z updates + 6 reductions, 2 grid barriers)",
                    "bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(ach / hbm, 3), "traffic": None,
                    "peak_source": f"{peak_kind} hbm_gbs",
                    "bytes_per_launch": b_it32, "ms_per_launch": round(km[2], 5),
                    "unit_of_work": "one CG iteration (the kernel loops over iterations)"}
    else:
        # the dominant kernel of the FP32 iteration: the larger of the two fused kernels
        dom = 0 if km[0] >= km[1] else 1
        if dom == 0:
            form = {0: "csr", 1: "rowclass", 2: "stencil"}[rc_mode]
            name = (f"cg_spmv<float> (w = A r, p = zc r + beta p, q = zc w + beta q, "
                    f"x += alpha p_old, (p,q), (r,r), (r,q), (q,q); FP32 CG iteration, {form} "
                    f"matrix form)")
            byt, ms_k = b_spmv32, km[0]
            key = f"cg_spmv<float>/{form}"
        else:
            name = "cg_update_r<float> (r -= alpha q, FP32 CG iteration, no reduction)"
            byt, ms_k = b_upd32, km[1]
            key = "cg_update_r<float>"
        ach = gbs(byt, ms_k)
        its_med = statistics.median(its)
        warm_ms = kwarm[dom]
        ach_warm = gbs(byt, warm_ms)
        iter_ms = kwarm[0] + kwarm[1]
        # achieved = algorithmic bytes over the kernel's launch time as it runs inside the
        # solve (replayed on the solver's own vectors, L2-warm); the cold launch (inputs
        # from HBM) is reported beside it
        roofline = {"kernel": name,
                    "bound": "hbm", "achieved": round(ach_warm, 1), "peak": hbm,
                    "unit": "GB/s", "frac": round(ach_warm / hbm, 3),
                    "traffic": profile_traffic(key),
                    "traffic_note": "dram__bytes_read + write of one launch in ncu's cold "
                                    "replay (profiles/); inside the solve the FP32 vectors "
                                    "and masks are L2-resident, so less comes from DRAM",
                    "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                    "l2_copy_gbs_measured": round(l2_gbs, 1) if l2_gbs else None,
                    "l2_frac": round(ach_warm / l2_gbs, 3) if l2_gbs else None,
                    "bytes_per_launch": byt, "ms_per_launch": round(warm_ms, 5),
                    "timing": "the two iteration kernels replayed 200 times back to back "
                              "on the solver's own vectors (as inside the timed solves), "
                              "CUDA events on the solver's stream; the FP32 vectors (8.4 MB "
                              "each) and the 4.2 MB of masks stay in L2, so the in-solve "
                              "bound is L2 (l2_frac) more than HBM",
                    "iteration_ms": round(iter_ms, 5),
                    "iterations": its_med,
                    "iterations_x_iteration_ms": round(its_med * iter_ms, 3),
                    "ms_per_step": round(mixed_ms, 3),
                    "consistent": bool(its_med * iter_ms <= mixed_ms),
                    "cold": {"ms_per_launch": round(ms_k, 5), "achieved": round(ach, 1),
                             "frac": round(ach / hbm, 3),
                             "timing": "CUDA events: 30 (256 MB read-only L2 flush, launch) "
                                       "pairs back to back minus the 30 flushes alone, so "
                                       "every launch reads its inputs from HBM with L2 clean "
                                       "and no idle-stream launch latency is counted"}}
    kernels = {
        "cg_persistent_f32_iter": {"ms": round(km[2], 5),
                                   "gbs": round(gbs(b_spmv32 + b_upd32, km[2]), 1) if km[2] else None},
        "cg_persistent_f64_iter": {"ms": round(k64[2], 5),
                                   "gbs": round(gbs(b_spmv64 + b_upd64, k64[2]), 1) if k64[2] else None},
        "cg_spmv_f32": {"ms": round(km[0], 5), "gbs": round(gbs(b_spmv32, km[0]), 1)},
        "cg_update_f32": {"ms": round(km[1], 5), "gbs": round(gbs(b_upd32, km[1]), 1)},
        "cg_spmv_f64": {"ms": round(k64[0], 5), "gbs": round(gbs(b_spmv64, k64[0]), 1)},
        "cg_update_f64": {"ms": round(k64[1], 5), "gbs": round(gbs(b_upd64, k64[1]), 1)},
        "spmv_f64_apply": {"ms": round(sp.value, 5), "gbs": round(gbs(b_apply, sp.value), 1),
                           "frac": round(gbs(b_apply, sp.value) / hbm, 3),
                           "form": {0: "CSR", 1: "row classes", 2: "stencil masks"}[rc_mode]},
        "spmv_f64_apply_csr": {"ms": round(sp_csr_seq.value, 5),
                               "gbs": round(gbs(b_apply_csr, sp_csr_seq.value), 1),
                               "frac": round(gbs(b_apply_csr, sp_csr_seq.value) / hbm, 3),
                               "timing": "50 launches back to back (inputs 217 MB > L2)",
                               "each_launch_after_l2_flush": {
                                   "ms": round(sp_csr.value, 5),
                                   "gbs": round(gbs(b_apply_csr, sp_csr.value), 1)}},
        # the whole mixed solve as FP32 iterations: algorithmic bytes of its iterations over
        # the solve's device time (refreshes, reductions and launch gaps included)
        "mixed_solve_effective": {
            "ms_per_iter": round(mixed_ms / max(1, statistics.median(its)), 5),
            "gbs": round(gbs((b_spmv32 + b_upd32) * statistics.median(its), mixed_ms), 1)},
    }

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            from oracle import oracle as O
            kind = "ref" if os.path.exists(O.REF_SO) else "port"
            full_ms, ref_iters, ref_code = reference_full(A, b, kind)
            cpu = {"value": round(full_ms, 1), "unit": "ms",
                   "cores": 1, "kind": "reference" if kind == "ref" else "port",
                   "sample": f"one complete Jacobi-PCG solve of this system by the reference "
                             f"from x0 = 0 to rtol 1e-8 ({ref_iters} iterations, code "
                             f"{ref_code}); serial solve path"}
        except Exception as exc:  # the baseline must not sink the GPU line
            cpu = {"value": None, "unit": "ms", "cores": 1, "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    # the other configurations of the path, compactly (one GPU only; about 30 s)
    workloads = None
    if rank == 0 and ws == 1 and not args.no_workloads:
        t0 = time.perf_counter()
        ref_its = fullsize_reference()
        p2, p2cpu = pcg2d_results(3, cpu=not args.no_cpu_baseline)
        if "p2d256_pcg" in ref_its:
            p2["reference_iterations"] = ref_its["p2d256_pcg"]
        workloads = {
            "pcg2d256": {"config": "2D 5-point 256x256, Jacobi-PCG rtol 1e-8, x0 = 0",
                         "gpu": p2, "cpu_baseline": p2cpu},
            "krylov96": {"config": "96^3 upwind convection-diffusion, Pe 0.1 and 10, weighted "
                                   "Jacobi 2/3, rtol 1e-8, GMRES restart fixed at 30 "
                                   "(gmres) or the reference's default 10-30 (gmresvar), "
                                   "Arnoldi by classical Gram-Schmidt with the "
                                   "reorthogonalisation delayed into the next step",
                         "results": krylov_results(96, 2, algs=("bicgstab", "gmres", "gmresvar"),
                                                   reference=ref_its)},
            "batch4096": batch_results(args, None, 0, 1, local, loop_sample=4),
            "adjoint64": adjoint_results(64, 2, fd_dirs=0),
        }
        workloads["wall_s"] = round(time.perf_counter() - t0, 1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(mixed_ms, 3), "unit": "ms", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(mixed_ms, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 Krylov iterations / f64 reliable updates", "data": "synthetic",
            "config": {"workload": f"3D Poisson 7-point {args.size}^3 (n={n}, nnz={nnz}), "
                                   f"Jacobi-PCG, FP64 rtol 1e-8, x0=0, b=A x*, x*~U[0,1)",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "L2 flushed between timed solves (256 MB read, leaving it "
                             "clean); kernel rooflines timed after the same flush (paired "
                             "flush + launch minus flush alone)",
                       "spmv_lanes_per_row": lanes,
                       "reliable_update_delta": args.delta,
                       "precision_mode": "MIXED_RELIABLE"},
            "fp64_ms": round(fp64_ms, 3), "mixed_over_fp64": round(mixed_ms / fp64_ms, 3),
            "step_ms": {"mixed": [round(t, 3) for t in times],
                        "fp64": [round(t, 3) for t in times64]},
            "csr_form": {"mixed_ms": round(csr_res[("mixed", False)][0], 3),
                         "fp64_ms": round(csr_res[("fp64", False)][0], 3),
                         "iterations": csr_res[("fp64", False)][1],
                         "col16_mixed_ms": round(csr_res[("mixed", True)][0], 3),
                         "col16_fp64_ms": round(csr_res[("fp64", True)][0], 3),
                         "note": "the same solves with the matrix in CSR form (no row-class "
                                 "or stencil-mask compression), as a general FASP++ matrix "
                                 "runs, with 32-bit column indices (the default) and, "
                                 "col16_*, with the opt-in 16-bit column offsets"},
            "restarted_refinement": {"ms": round(restarted_ms, 3),
                                     "over_fp64": round(restarted_ms / fp64_ms, 3),
                                     "inner_rel_tol": args.inner_tol,
                                     "inner_total": int(statistics.median(itsR)),
                                     "outer": outerR},
            "iterations": {"mixed_fp32": int(statistics.median(its)),
                           "mixed_fp64_refreshes": outer, "fp64": int(statistics.median(its64))},
            "accuracy": {"mixed_rel_residual": acc_mixed[0], "mixed_err_vs_fp64_1e-13": acc_mixed[1],
                         "fp64_rel_residual": acc_fp64[0], "fp64_err_vs_fp64_1e-13": acc_fp64[1],
                         "e2e_err_vs_fp64_1e-13": e2e_err},
            "spmv_gbs": kernels["spmv_f64_apply_csr"]["gbs"],
            "matrix_form": {"mode": {0: "CSR", 1: "row classes", 2: "stencil masks"}[rc_mode],
                            "classes": rc_classes, "table_entries": rc_entries,
                            "stencil_offsets": rc_stencil},
            "roofline": roofline, "kernels": kernels,
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": 2 * 8 * n,
                    "d2h_bytes_per_step": 8 * n},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "workloads": workloads,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


M_BINS = np.linspace(16, 129, 9)  # strata of the batch's grid sizes m for the loop sample


def batch_results(args, dist=None, rank=0, ws=1, local=0, loop_sample=8):
    """The batched workload: 4,096 shifted 2D Poisson systems (m ~ U{16..128}, sigma ~
    U[0,1]), 4 right-hand sides each (b ~ N(0,1)), Jacobi-PCG to rtol 1e-8. Under torchrun
    every rank builds and solves only its share of the systems (shard.partition: LPT by
    nnz, the same on every rank, no data-path collective) in one persistent launch; the
    batch's time is the slowest rank's. On one GPU also the loop of per-system FP64 GPU
    solves it replaces, timed on a stratified sample (loop_sample systems from each of 8
    bins of m, all 4 right-hand sides) and scaled per bin by the bin's system count."""
    from faspxx_b200 import batch as BT
    from faspxx_b200 import capi, problems as P, shard as S, sol
    count = args.batch_count
    ms, sig, rhs = P.batch_systems(count=count, nrhs=4, seed=42)
    work = 5 * ms.astype(np.int64) ** 2
    shards = S.partition(work, ws)
    mine = shards[rank]
    mats = [P.poisson2d(int(ms[i]), shift=float(sig[i])) for i in mine]
    B = BT.Batch(mats, nrhs=4, device=local)
    b = np.zeros((4, B.N))
    for k, i in enumerate(mine):
        b[:, B.sys_row[k]:B.sys_row[k + 1]] = rhs[i]
    db = BT._Dev(np.ascontiguousarray(b))
    shape64, _ = B.autotune(b, precision=capi.FP64)
    res = {}
    steps = max(1, min(args.steps, 5))
    for name, prec, tol in (("fp64", capi.FP64, 1e-4), ("mixed", capi.MIXED_RELIABLE, 1e-2)):
        for _ in range(2):
            B.solve(db, relTol=1e-8, precision=prec, innerRelTol=tol)
        t = []
        for _ in range(steps):
            barrier(dist)
            x, it, rr, m = B.solve(db, relTol=1e-8, precision=prec, innerRelTol=tol)
            t.append(m)
        res[name] = (dist_max(dist, statistics.mean(t)), int(it.sum()), float(rr.max()))
    local_res = {"systems": mine.tolist(), "iters": it.tolist(), "rows": int(B.N)}
    gathered = S.gather_results(dist, rank, ws, local_res)
    out = {"systems": count, "rows_total": int(sum(int(m) ** 2 for m in ms)),
           "shape": list(shape64), "ranks": ws,
           "fp64_ms": round(res["fp64"][0], 3), "mixed_ms": round(res["mixed"][0], 3),
           "iterations_mixed_this_rank": res["mixed"][1],
           "max_rel_residual": {"fp64": res["fp64"][2], "mixed": res["mixed"][2]}}
    if rank == 0 and gathered:
        out["systems_gathered"] = sum(len(g["systems"]) for g in gathered)
        out["imbalance"] = round(S.imbalance(work, shards), 4)
    if ws == 1:
        # the loop of per-system FP64 GPU solves (device-driven CG, setup excluded), stratified
        rng = np.random.default_rng(1)
        loop_total, sampled = 0.0, 0
        for lo, hi in zip(M_BINS[:-1], M_BINS[1:]):
            cand = np.nonzero((ms >= lo) & (ms < hi))[0]
            if len(cand) == 0:
                continue
            pick = rng.choice(cand, size=min(loop_sample, len(cand)), replace=False)
            tsum = 0.0
            for k in pick:
                Mk = sol.MAT(P.poisson2d(int(ms[k]), shift=float(sig[k])))
                s = sol.configure("cg", maxIter=5000, relTol=1e-8, absTol=0.0, pcd="jacobi",
                                  pcdWeight=1.0, pcdIter=1)
                s.Setup(Mk)
                n = int(ms[k]) ** 2
                dbk, dxk = sol.DVec(n), sol.DVec(n)
                for j in range(4):
                    dbk.set(rhs[k][j])
                    dxk.Zero()
                    capi.lib.fasp_gpu_synchronize()
                    t0 = time.perf_counter()
                    s.Solve(dbk, dxk)
                    tsum += (time.perf_counter() - t0) * 1e3
            loop_total += tsum / len(pick) * len(cand)
            sampled += len(pick)
        out["loop_per_system_fp64_ms"] = round(loop_total, 1)
        out["loop_sample"] = (f"{sampled} systems (up to {loop_sample} from each of 8 bins of m "
                              f"over [16, 128]) x 4 RHS timed (host wall clock per solve), "
                              f"each bin's mean scaled by its system count")
        out["speedup_vs_loop"] = {"fp64": round(loop_total / res["fp64"][0], 1),
                                  "mixed": round(loop_total / res["mixed"][0], 1)}
    return out


def run_batch(args):
    """--workload batch: the batched workload on its own JSON line; under torchrun the
    systems shard across ranks (strong scaling: the whole batch's time)."""
    ws, rank, local = dist_env()
    dist = dist_init(ws)
    from faspxx_b200 import capi
    capi.init(local)
    r = batch_results(args, dist, rank, ws, local)
    if rank == 0:
        line = {"metric": "Batched Jacobi-PCG, 4096 uneven systems x 4 RHS to rtol 1e-8",
                "value": r["mixed_ms"], "unit": "ms", "n_gpus": ws, "steps": args.steps,
                "warmup": 2, "ms_per_step": r["mixed_ms"], "higher_is_better": False,
                "scaling": "strong", "vs_baseline": None,
                "dtype": "f32 Krylov iterations / f64 reliable updates", "data": "synthetic",
                "config": {"workload": "4096 systems, 2D 5-point m~U{16..128} + sigma I, "
                                       "sigma~U[0,1], 4 RHS b~N(0,1), Jacobi-PCG rtol 1e-8",
                           "parallelism": f"systems sharded over {ws} ranks (LPT by nnz)"
                                          if ws > 1 else "single GPU"},
                "results": r}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _time_solve(s, db, dx, reps, warm=2, flush=None):
    """Mean device time (ms) of reps solves from x0 = 0 (after warm untimed ones)."""
    ts = []
    for i in range(warm + reps):
        dx.Zero()
        if flush is not None:
            flush.Norm2()  # read-only: evicts L2 without leaving dirty lines
        code = s.Solve(db, dx)
        if i >= warm:
            ts.append(s.LastTimeMs())
    return statistics.mean(ts), code


def krylov_results(N, steps, algs=("bicgstab", "gmres", "fgmres"), reference=None, orth=None):
    """Nonsymmetric 3D convection-diffusion -Laplace(u) + beta.grad(u) on N^3 (first-order
    upwind, direction (1, 0.5, 0.25), cell Peclet 0.1 and 10), b = A x* with x* ~ U[-1,1)
    (seed 42), x0 = 0, rtol 1e-8, weighted Jacobi (omega = 2/3, one sweep), GMRES/FGMRES with
    a fixed restart of 30 and (gmresvar) GMRES with the reference's default variable restart
    between 10 and 30: FP64, FP32 inner iterations inside FP64 refinement (FP64 residual,
    update and Hessenberg/Givens least squares) and, for BiCGStab, FP32 iterations with FP64
    reliable updates. reference: the reference's iteration counts by case name,
    where recorded. orth: the GMRES/FGMRES Gram-Schmidt variant (None: the library's
    default)."""
    from faspxx_b200 import capi, problems as P, sol
    flush = sol.DVec(32 << 20)
    rows = []
    for pe, tag in ((0.1, "pe01"), (10.0, "pe10")):
        A = P.convdiff3d(N, pe)
        xs = P.seeded_uniform(A.nrow, 42, -1.0, 1.0)
        b = A.matvec(xs)
        M = sol.MAT(A)
        M.Autotune()
        db, dx = sol.DVec.from_numpy(b), sol.DVec(A.nrow)
        for alg in algs:
            res = {}
            precs = ("fp64", "mixed") + (("reliable",) if alg == "bicgstab" else ())
            for prec in precs:
                kw = dict(maxIter=5000, relTol=1e-8, absTol=0.0, pcd="jacobi",
                          pcdWeight=2.0 / 3.0, pcdIter=1)
                if alg in ("gmres", "fgmres"):
                    kw.update(restart=30, maxRestart=30, minRestart=30)
                # gmresvar: the reference's default variable restart (10 to 30)
                s = sol.configure("gmres" if alg == "gmresvar" else alg, **kw)
                if orth is not None and alg in ("gmres", "gmresvar", "fgmres"):
                    s.SetOrth(orth)
                if prec == "mixed":
                    s.SetPrecision(capi.MIXED, innerRelTol=1e-4, maxOuter=50)
                elif prec == "reliable":
                    s.SetPrecision(capi.MIXED_RELIABLE, innerRelTol=1e-3)
                s.Setup(M)
                ms, code = _time_solve(s, db, dx, steps, flush=flush)
                x = dx.numpy()
                rel = float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b))
                # code 0 at maxIter is the reference's convention (FGMRES.cxx:226 tests
                # numIter > maxIter): say plainly whether the tolerance was met
                res[prec] = {"ms": round(ms, 3), "code": code, "iters": s.GetIterations(),
                             "outer": s.info.outerIter if prec != "fp64" else None,
                             "rel_residual": rel,
                             "converged": bool(rel <= 1.01e-8),
                             "err_vs_xstar": float(np.linalg.norm(x - xs) / np.linalg.norm(xs))}
            row = {"peclet": pe, "solver": alg, **{k: v for k, v in res.items()},
                   "mixed_over_fp64": round(res["mixed"]["ms"] / res["fp64"]["ms"], 3)}
            if "reliable" in res:
                row["reliable_over_fp64"] = round(res["reliable"]["ms"] / res["fp64"]["ms"], 3)
            key = f"cd{N}_{tag}_{alg}"
            if reference and key in reference:
                row["reference_iterations"] = reference[key]
            rows.append(row)
    return rows


def fullsize_reference():
    """Iteration counts of the reference on the full-size systems, recorded from the reference
    compiled from its own sources (tests/golden/fullsize.json); {} when absent."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "fullsize.json")) as f:
            d = json.load(f)
    except OSError:
        return {}
    return {k: v["iters"] for k, v in d.items() if "iters" in v}


def run_krylov(args):
    """--workload krylov96: BiCGStab / GMRES(30) / FGMRES(30) at 96^3, FP64 and mixed."""
    from faspxx_b200 import capi, problems as P, sol
    capi.init(0)
    N = args.size if args.size != N_GRID else 96
    if args.profile:
        # for ncu: one 60-iteration FP64 solve of BiCGStab and of GMRES(30) at Pe 0.1, then
        # one of BiCGStab with FP32 iterations and reliable updates
        A = P.convdiff3d(N, 0.1)
        b = A.matvec(P.seeded_uniform(A.nrow, 42, -1.0, 1.0))
        M = sol.MAT(A)
        if args.lanes:
            M.SetLanes(args.lanes)
        db, dx = sol.DVec.from_numpy(b), sol.DVec(A.nrow)
        for alg in ("bicgstab", "gmres", "bicgstab-reliable"):
            kw = dict(maxIter=60, relTol=1e-8, absTol=0.0, pcd="jacobi", pcdWeight=2.0 / 3.0,
                      pcdIter=1)
            if alg == "gmres":
                kw.update(restart=30, maxRestart=30, minRestart=30)
            s = sol.configure(alg.split("-")[0], **kw)
            if alg == "gmres" and args.orth != "default":
                s.SetOrth(getattr(capi, "ORTH_" + args.orth.upper()))
            if alg == "bicgstab-reliable":
                s.SetPrecision(capi.MIXED_RELIABLE, innerRelTol=1e-2)
            s.Setup(M)
            dx.Zero()
            code = s.Solve(db, dx)
            print(f"profile {alg} code {code} iterations {s.GetIterations()} "
                  f"{s.LastTimeMs():.3f} ms")
        return 0
    orth = None if args.orth == "default" else getattr(capi, "ORTH_" + args.orth.upper())
    rows = krylov_results(N, args.steps, algs=("bicgstab", "gmres", "gmresvar", "fgmres"),
                          reference=fullsize_reference(), orth=orth)
    total_mixed = sum(r["mixed"]["ms"] for r in rows)
    line = {"metric": "Time to rtol 1e-8, 96^3 convection-diffusion, BiCGStab / GMRES(30) / "
                      "FGMRES(30): FP32-inner refinement vs FP64",
            "value": round(total_mixed, 3), "unit": "ms (sum of the six mixed solves)",
            "n_gpus": 1, "steps": args.steps, "warmup": 2, "higher_is_better": False,
            "dtype": "f32 inner / f64 refinement", "data": "synthetic",
            "config": {"workload": f"{N}^3 upwind convection-diffusion, Pe 0.1 and 10, "
                                   "weighted Jacobi 2/3, x0=0, b=A x*, x*~U[-1,1)",
                       "arnoldi": "GMRES: " + (args.orth if args.orth != "default" else "dcgs2")
                                  + "; FGMRES: cgs2" if args.orth != "mgs" else "mgs",
                       "l2": "L2 flushed between timed solves"},
            "results": rows}
    print(json.dumps(line))
    return 0


def adjoint_results(N, steps, fd_dirs):
    """Differentiable solve of -div(kappa grad u) = b on 64^3 (kappa = exp(N(0,1)) per cell,
    harmonic face averages; b ~ N(0,1)); loss 0.5 ||x - x_t||^2 (x_t ~ N(0,1)). Forward CG to
    rtol 1e-10 (Jacobi), backward the adjoint CG on the exact transpose + the sampled outer
    product. FP64 and FP32-iteration (reliable-update) variants; gradients checked by central
    differences (eps 1e-6) along 32 seeded random directions and against the FP64 gradient."""
    from faspxx_b200 import capi, problems as P, sol
    lib = capi.lib
    rng = np.random.default_rng(42)
    kappa = np.exp(rng.standard_normal(N ** 3))
    A = P.vardiff3d(N, kappa)
    n, nnz = A.nrow, A.nnz
    b = rng.standard_normal(n)
    xt = rng.standard_normal(n)
    db, dx, dg, dlam = sol.DVec.from_numpy(b), sol.DVec(n), sol.DVec(n), sol.DVec(n)
    dA = sol.DVec(nnz)

    def make(M, prec):
        s = sol.configure("cg", maxIter=20000, relTol=1e-10, absTol=0.0, pcd="jacobi",
                          pcdWeight=1.0, pcdIter=1)
        if prec != capi.FP64:
            s.SetPrecision(prec, innerRelTol=1e-2)
        s.Setup(M)
        return s

    out = {}
    M = sol.MAT(A)
    for name, prec in (("fp64", capi.FP64), ("fp32_iter", capi.MIXED_RELIABLE)):
        s = make(M, prec)
        fwd, bwd, outer_ms = [], [], []
        info = capi.Info()
        for i in range(2 + steps):
            dx.Zero()
            s.Solve(db, dx)
            f = s.LastTimeMs()
            x = dx.numpy()
            dg.set(x - xt)
            dlam.Zero()  # lambda0 = 0
            lib.fasp_gpu_synchronize()
            capi.check(lib.fasp_gpu_solver_solve_adjoint(s.h, dg.ptr, dlam.ptr, C.byref(info)),
                       "adjoint")
            bt = s.LastTimeMs()
            lib.fasp_gpu_synchronize()
            t0 = time.perf_counter()
            capi.check(lib.fasp_gpu_mat_sampled_outer(M.h, dlam.ptr, dx.ptr, -1.0, dA.ptr),
                       "sampled_outer")
            lib.fasp_gpu_synchronize()
            t1 = time.perf_counter()
            if i >= 2:
                fwd.append(f)
                bwd.append(bt)
                outer_ms.append((t1 - t0) * 1e3)
        out[name] = {"forward_ms": round(statistics.mean(fwd), 3),
                     "adjoint_ms": round(statistics.mean(bwd), 3),
                     "outer_ms_wall": round(statistics.mean(outer_ms), 4),
                     "iters_forward": s.GetIterations(), "adjoint_iters": info.numIter,
                     "grad_b": dlam.numpy(), "grad_A": dA.numpy(), "x": dx.numpy()}
    g64b, g64A = out["fp64"]["grad_b"], out["fp64"]["grad_A"]
    rel = lambda u, v: float(np.linalg.norm(u - v) / np.linalg.norm(v))  # noqa: E731
    # central differences of the FP64 loss along 32 random (b, A-values) directions
    eps = 1e-6
    s64 = make(M, capi.FP64)
    x0 = out["fp64"]["x"]

    def loss(vals, bb):
        Mp = sol.MAT(P.CSRMatrix(n, n, A.rowPtr, A.colInd, vals))
        sp = make(Mp, capi.FP64)
        dbb = sol.DVec.from_numpy(bb)
        dxx = sol.DVec(n)
        sp.Solve(dbb, dxx)
        xx = dxx.numpy()
        return 0.5 * float(np.dot(xx - xt, xx - xt))

    errs = []
    drng = np.random.default_rng(7)
    for _ in range(fd_dirs):
        dbdir = drng.standard_normal(n)
        dAdir = drng.standard_normal(nnz) * np.abs(A.values)
        lp = loss(A.values + eps * dAdir, b + eps * dbdir)
        lm = loss(A.values - eps * dAdir, b - eps * dbdir)
        fd = (lp - lm) / (2 * eps)
        an = float(np.dot(g64b, dbdir) + np.dot(g64A, dAdir))
        errs.append(abs(fd - an) / max(abs(an), 1e-300))
    del s64, x0
    out_d = {"n": n, "nnz": nnz,
             "fp64": {k: v for k, v in out["fp64"].items() if not k.startswith(("grad", "x"))},
             "fp32_iter": {k: v for k, v in out["fp32_iter"].items()
                           if not k.startswith(("grad", "x"))},
             "fp32_iter_grad_rel_err_vs_fp64": {"b": rel(out["fp32_iter"]["grad_b"], g64b),
                                                 "A": rel(out["fp32_iter"]["grad_A"], g64A)},
             "central_difference": {"directions": fd_dirs, "eps": eps,
                                    "max_rel_err": max(errs) if errs else None,
                                    "median_rel_err": statistics.median(errs) if errs else None}}
    # against the reference's own gradient (recorded from the reference compiled from its
    # sources: forward CG, adjoint CG on its MAT::TransInPlace, -lambda_i x_j), projected on
    # the same 32 seeded directions
    try:
        z = np.load(os.path.join(ROOT, "tests", "golden", "fullsize.npz"))
        proj_ref = z["vd64_adjoint__proj"]
        drng = np.random.default_rng(7)
        proj = np.array([float(np.dot(g64b, drng.standard_normal(n)) +
                               np.dot(g64A, drng.standard_normal(nnz))) for _ in range(32)])
        if N == 64:
            out_d["fp64_grad_vs_reference_projections_max_rel_err"] = float(
                np.max(np.abs(proj - proj_ref) / np.abs(proj_ref)))
    except (OSError, KeyError):
        pass
    return out_d


def run_adjoint(args):
    """--workload adjoint64: the differentiable 64^3 solve on its own JSON line."""
    from faspxx_b200 import capi
    capi.init(0)
    N = args.size if args.size != N_GRID else 64
    r = adjoint_results(N, args.steps, args.fd_dirs)
    line = {"metric": "Differentiable 64^3 variable-coefficient solve: forward + adjoint time, "
                      "gradient agreement",
            "value": round(r["fp64"]["forward_ms"] + r["fp64"]["adjoint_ms"], 3),
            "unit": "ms (FP64 forward + adjoint)", "n_gpus": 1, "steps": args.steps,
            "warmup": 2, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{N}^3 -div(kappa grad u), kappa=exp(N(0,1)), "
                                   f"n={r['n']}, nnz={r['nnz']}, CG rtol 1e-10, Jacobi"},
            "results": r}
    print(json.dumps(line))
    return 0


def pcg2d_results(steps, cpu=True):
    """2D 5-point Poisson on a 256 x 256 grid (n = 65,536, nnz = 326,656), x* ~ U[0,1) (seed
    42), b = A x*, x0 = 0, Jacobi-PCG to rtol 1e-8, max 2000 iterations: the reference's PCG
    example at its own size, device-driven FP64 and FP32-iteration (reliable-update) CG; with
    cpu, one complete solve by the reference (compiled from its sources) on the host."""
    from faspxx_b200 import capi, problems as P, sol
    A = P.poisson2d(256)
    xs = P.seeded_uniform(A.nrow, 42)
    b = A.matvec(xs)
    M = sol.MAT(A)
    M.Autotune()
    db, dx = sol.DVec.from_numpy(b), sol.DVec(A.nrow)
    flush = sol.DVec(32 << 20)
    res = {}
    for name, prec in (("fp64", capi.FP64), ("mixed", capi.MIXED_RELIABLE)):
        s = sol.configure("cg", maxIter=2000, relTol=1e-8, absTol=0.0, pcd="jacobi",
                          pcdWeight=1.0, pcdIter=1)
        if prec != capi.FP64:
            s.SetPrecision(prec, innerRelTol=1e-2)
        s.Setup(M)
        ms, code = _time_solve(s, db, dx, steps, flush=flush)
        x = dx.numpy()
        res[name] = {"ms": round(ms, 3), "code": code, "iters": s.GetIterations(),
                     "rel_residual": float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)),
                     "err_vs_xstar": float(np.linalg.norm(x - xs) / np.linalg.norm(xs))}
    cpu_res = None
    if cpu:
        from oracle import oracle as O
        kind = "ref" if os.path.exists(O.REF_SO) else "port"
        full_ms, iters, code = reference_full(A, b, kind)
        cpu_res = {"value": round(full_ms, 2), "unit": "ms", "cores": 1,
                   "kind": "reference" if kind == "ref" else "port", "iterations": iters,
                   "sample": "one complete Jacobi-PCG solve of the same system on the host"}
    return res, cpu_res


def run_pcg2d(args):
    """--workload pcg2d256: the reference's PCG example at 256 x 256."""
    from faspxx_b200 import capi
    capi.init(0)
    res, cpu = pcg2d_results(args.steps, cpu=not args.no_cpu_baseline)
    line = {"metric": "Time to rtol 1e-8, 2D Poisson 256x256 Jacobi-PCG",
            "value": res["fp64"]["ms"], "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": 2, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "2D 5-point 256x256 (n=65536, nnz=326656), Jacobi-PCG, "
                                   "x0=0, b=A x*, x*~U[0,1)"},
            "results": res, "cpu_baseline": cpu}
    print(json.dumps(line))
    return 0


def run_matfree(args):
    """The reference's matrix-free example (example/TestMatFree.cxx:178-255): CG without a
    preconditioner on the 2D 5-point operator of the (dim-1)^2 interior grid, dim = 16 ...
    512, relTol 1e-8, absTol 1e-12, x0 = 0.25, its right-hand side (u = sin(pi x) sin(pi y)).
    GPU: the matrix-free grid operator (no stored matrix) and, at dim 512, the stored CSR
    matrix in its stencil-mask form. CPU: the reference example itself (built from the
    reference sources into oracle/_ref), its own wall-clock timing of each CG solve."""
    import re
    from faspxx_b200 import capi, problems as P, sol
    from oracle import oracle as O
    capi.init(0)
    five = [((0, -1), -1.0), ((-1, 0), -1.0), ((0, 0), 4.0), ((1, 0), -1.0), ((0, 1), -1.0)]
    res = {}
    for dim in (16, 32, 64, 128, 256, 512):
        n = (dim - 1) ** 2
        b = sol.DVec.from_numpy(O.matfree_rhs(dim))
        x = sol.DVec(n)
        x0 = np.full(n, 0.25)
        forms = [("grid", sol.MAT.Stencil((dim - 1, dim - 1), five))]
        if dim == 512:
            forms.append(("stored", sol.MAT(P.poisson2d(dim - 1))))
        for form, M in forms:
            s = sol.configure("cg", maxIter=10000, restart=20, relTol=1e-8, absTol=1e-12)
            s.Setup(M)
            ts = []
            for i in range(args.warmup + args.steps):
                x.set(x0)
                if s.Solve(b, x) != 0:
                    raise RuntimeError("matrix-free CG failed")
                if i >= args.warmup:
                    ts.append(s.LastTimeMs())
            h = 1.0 / dim
            k = np.arange(1, dim)
            u = np.outer(np.sin(np.pi * k * h), np.sin(np.pi * k * h)).ravel()
            err = float(np.sqrt(np.sum((x.numpy() - u) ** 2) * h * h))
            key = str(dim) if form == "grid" else f"{dim}_stored_matrix"
            res[key] = {"ms": round(statistics.mean(ts), 4), "iters": s.GetIterations(),
                        "norm2": s.GetNorm2(), "l2_error": err}
    cpu = None
    exe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "_ref",
                       "test_matfree")
    if not args.no_cpu_baseline and os.path.exists(exe):
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            out = subprocess.run([exe], cwd=d, capture_output=True, text=True,
                                 timeout=600).stdout
        cpu = {}
        for block in out.split("dim = ")[1:]:
            dim = int(block.split(",")[0])
            cpu[str(dim)] = {"ms": float(re.search(r"costs\s+([0-9.eE+-]+)ms", block).group(1)),
                             "iters": int(re.search(r"NumIter\s*:\s*(\d+)", block).group(1))}
    line = {"metric": "Time of the matrix-free CG solve, reference example TestMatFree "
                      "(2D Poisson, dim 512: n = 261,121)",
            "value": res["512"]["ms"], "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "dtype": "f64",
            "data": "the example's own right-hand side",
            "config": {"workload": "example/TestMatFree.cxx: 5-point operator on the "
                                   "(dim-1)^2 interior grid, CG without preconditioner, "
                                   "rtol 1e-8, atol 1e-12, x0 = 0.25, dim 16..512"},
            "results": res,
            "cpu_baseline": None if not cpu else {
                "value": cpu["512"]["ms"], "unit": "ms", "cores": 1, "kind": "reference",
                "sample": "the reference example's own timing of each CG solve",
                "per_dim": cpu}}
    print(json.dumps(line))
    return 0


def _interp_trilinear(nf: int):
    """Trilinear prolongation from the ((nf-1)/2)^3 grid to nf^3 (x fastest), as CSR arrays."""
    import scipy.sparse as sp
    nc = (nf - 1) // 2
    rows, cols, vals = [], [], []
    for i in range(nf):
        if i % 2 == 1:
            rows.append(i), cols.append((i - 1) // 2), vals.append(1.0)
        else:
            if i // 2 - 1 >= 0:
                rows.append(i), cols.append(i // 2 - 1), vals.append(0.5)
            if i // 2 < nc:
                rows.append(i), cols.append(i // 2), vals.append(0.5)
    p1 = sp.csr_matrix((vals, (rows, cols)), shape=(nf, nc))
    p3 = sp.kron(p1, sp.kron(p1, p1, format="csr"), format="csr")
    p3.sort_indices()
    return p3


def run_mg(args):
    """Geometric multigrid on the 3D 7-point Poisson matrix at 127^3 (n = 2,048,383): the
    headline's system at the nearest size that coarsens to a point (127 -> 63 -> 31 -> 15 ->
    7 -> 3), trilinear prolongation, restriction = its transpose and Galerkin coarse
    operators formed on the GPU (MAT::Mult), Jacobi V(2,2) cycles with 40 sweeps on 3^3.
    Reported: the setup (transposes and Galerkin products), MG-preconditioned CG and plain MG
    to rtol 1e-8, against Jacobi-PCG in FP64 and in mixed precision on the same system."""
    from faspxx_b200 import capi, problems as P, sol
    capi.init(0)
    nf = 127
    A = P.poisson3d(nf)
    xs = P.seeded_uniform(A.nrow, 42)
    b = A.matvec(xs)
    M = sol.MAT(A)
    Ps, keep = [], []
    f = nf
    t0 = time.perf_counter()
    while f > 3:
        p3 = _interp_trilinear(f)
        Ps.append(sol.MAT(P.CSRMatrix(p3.shape[0], p3.shape[1], p3.indptr.astype(np.uint32),
                                      p3.indices.astype(np.uint32), p3.data.astype(np.float64))))
        f = (f - 1) // 2
    build_s = time.perf_counter() - t0
    L = len(Ps)
    mgkw = dict(mgLevels=L, mgCycles=1, mgSmooth=dict(maxIter=2, minIter=2, weight=2.0 / 3.0),
                mgCoarse=dict(maxIter=40, minIter=40, weight=2.0 / 3.0))
    db, dx = sol.DVec.from_numpy(b), sol.DVec(A.nrow)
    flush = sol.DVec(32 << 20)
    res = {}
    configs = [("mg_pcg", sol.configure("cg", maxIter=200, relTol=1e-8, absTol=0.0, pcd="mg",
                                        pcdIter=1, **mgkw)),
               ("mg", sol.configure("mg", maxIter=200, relTol=1e-8, absTol=0.0, **mgkw)),
               ("jacobi_pcg_fp64", sol.configure("cg", maxIter=2000, relTol=1e-8, absTol=0.0,
                                                 pcd="jacobi", pcdIter=1)),
               ("jacobi_pcg_mixed", sol.configure("cg", maxIter=2000, relTol=1e-8, absTol=0.0,
                                                  pcd="jacobi", pcdIter=1))]
    configs[3][1].SetPrecision(capi.MIXED_RELIABLE, innerRelTol=1e-2)
    for name, s in configs:
        if name.startswith("mg"):
            s.transfers = {l: (Ps[l], None, None) for l in range(L)}
        lib = capi.lib
        lib.fasp_gpu_synchronize()
        t0 = time.perf_counter()
        s.Setup(M)
        lib.fasp_gpu_synchronize()
        setup_ms = (time.perf_counter() - t0) * 1e3
        ms, code = _time_solve(s, db, dx, args.steps, flush=flush)
        x = dx.numpy()
        res[name] = {"ms": round(ms, 3), "setup_ms": round(setup_ms, 1), "code": code,
                     "iters": s.GetIterations(),
                     "rel_residual": float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b))}
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        kind = "ref" if os.path.exists(O.REF_SO) else "port"
        per_iter, _ = reference_sample(A, b, args.ref_sample, kind)
        cpu = {"value": round(per_iter * res["jacobi_pcg_fp64"]["iters"], 1), "unit": "ms",
               "cores": 1, "kind": "reference" if kind == "ref" else "port",
               "sample": f"{args.ref_sample} Jacobi-PCG iterations of the reference on this "
                         "system, scaled by the FP64 iteration count (the reference's MG "
                         "cannot use transfer operators)"}
    line = {"metric": "Time to rtol 1e-8, 3D Poisson 127^3: MG-preconditioned CG (V(2,2), "
                      "Galerkin hierarchy formed on the GPU)",
            "value": res["mg_pcg"]["ms"], "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": 2, "higher_is_better": False, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "3D 7-point 127^3 (n=2048383), b=A x*, x*~U[0,1), x0=0; "
                                   f"{L} coarse levels, trilinear P, R = P^T, Galerkin "
                                   "R A P, Jacobi 2/3 V(2,2), 40 sweeps on 3^3",
                       "l2": "L2 flushed between timed solves",
                       "prolongations_built_on_host_s": round(build_s, 2)},
            "results": res, "cpu_baseline": cpu}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=N_GRID)
    ap.add_argument("--inner-tol", type=float, default=1e-4,
                    help="inner tolerance of the restarted-refinement variant")
    ap.add_argument("--delta", type=float, default=1e-2,
                    help="reliable-update factor of the headline mixed solve")
    ap.add_argument("--ref-sample", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-workloads", action="store_true",
                    help="leave out the other configurations' compact block")
    ap.add_argument("--lanes", type=int, default=0, help="force SpMV lanes per row")
    ap.add_argument("--orth", choices=["default", "cgs2", "dcgs2", "mgs"], default="default",
                    help="krylov96: the GMRES/FGMRES Gram-Schmidt variant")
    ap.add_argument("--profile", action="store_true",
                    help="short runs for ncu: each fused CG kernel 4 times (poisson128), or "
                         "one 60-iteration BiCGStab and GMRES(30) solve (krylov96)")
    ap.add_argument("--form", choices=["auto", "csr"], default="auto",
                    help="poisson128: matrix form of the solves (csr: plain CSR, as a general "
                         "matrix; auto: the compressed form the matrix admits)")
    ap.add_argument("--profile-solve", action="store_true",
                    help="poisson128: three mixed solves only (for an ncu launch list)")
    ap.add_argument("--profile-apply", action="store_true",
                    help="poisson128: a few FP64 MAT::Apply launches only (for ncu)")
    ap.add_argument("--workload", choices=["poisson128", "batch", "krylov96", "adjoint64",
                                           "pcg2d256", "matfree", "mg127"],
                    default="poisson128")
    ap.add_argument("--fd-dirs", type=int, default=32)
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--batch-sample", type=int, default=256)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "krylov96":
        return run_krylov(args)
    if args.workload == "adjoint64":
        return run_adjoint(args)
    if args.workload == "pcg2d256":
        return run_pcg2d(args)
    if args.workload == "matfree":
        return run_matfree(args)
    if args.workload == "mg127":
        return run_mg(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
