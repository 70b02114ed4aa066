"""Record the reference's results at the workloads' full sizes (tests/golden/fullsize.*).

Run in a container that has the reference compiled into oracle/_ref (``make -C oracle``);
the GPU box only reads the outputs. For each case the compiled reference
(oracle/_ref/liboracle_ref.so) and the C restatement (oracle/liboracle_port.so) solve the
same system; the script requires that both return the same code, iteration count, norms
and solution bit for bit, so the restatement's full-precision residual history is the
reference's (the reference itself prints 6 significant digits, which are cross-checked).

Stored per case (the solutions are too large to commit whole): code, iterations, norms,
the full-precision residual history, the reference's printed history, the solution at
8,192 seeded positions, its 2-norm and sum, and the case's sensitivity envelope: the same
algorithm (the restatement) rerun four times with every entry of b moved by one ulp up or
down (four seeds), the iteration counts, the largest solution difference and, per
iteration, the largest history deviation.
A GPU that sums in another order perturbs every step by about that much, so the envelope
shows how closely any reordered implementation can follow the reference on the case.
Cases:

* ``p2d256_pcg``  -- 2D 5-point Poisson 256x256, Jacobi-PCG (weight 1, one sweep), rtol 1e-8;
* ``p3d128_pcg``  -- 3D 7-point Poisson 128^3, the same solver (the benchmark's system);
* ``cd96_pe{01,10}_{bicgstab,gmres}`` -- 96^3 upwind convection-diffusion, weighted Jacobi
  2/3, rtol 1e-8, GMRES(30) with a fixed restart;
* ``cd96_pe{01,10}_fgmres300`` -- FGMRES(30), its first 300 iterations;
* ``cd96_pe{01,10}_gmresvar`` -- GMRES with the reference's default variable restart;
* ``vd64_adjoint`` -- 64^3 variable-coefficient diffusion, forward CG to rtol 1e-10, the
  adjoint CG on MAT::TransInPlace(A) (the reference's transpose), dL/db = lambda and
  dL/dA_k = -lambda_row(k) x_col(k); stored as projections on 32 seeded directions plus
  8,192 sampled entries of each gradient;
* ``batch4096`` -- the 4,096-system batch: the reference's Jacobi-PCG iteration count and
  solution samples for a stratified sample of 64 systems (4 right-hand sides each).

    python tests/golden/make_fullsize.py [--only NAME ...] [--jobs J]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NSAMPLE = 8192
ENV_SEEDS = (1, 2, 3, 4)
SYN = dict(minIter=0, absTol=0.0)
JAC1 = dict(pcd="jacobi", pcdWeight=1.0, pcdIter=1)
JAC23 = dict(pcd="jacobi", pcdWeight=2.0 / 3.0, pcdIter=1)
GM30 = dict(restart=30, maxRestart=30, minRestart=30)


def solver_cases() -> dict:
    """name -> (matrix spec, alg, rhs kind, solver keywords)."""
    C = {"p2d256_pcg": (("poisson2d", 256), "cg", "xstar01",
                        dict(SYN, maxIter=2000, relTol=1e-8, **JAC1)),
         "p3d128_pcg": (("poisson3d", 128), "cg", "xstar01",
                        dict(SYN, maxIter=3000, relTol=1e-8, **JAC1))}
    for tag, pe in (("pe01", 0.1), ("pe10", 10.0)):
        C[f"cd96_{tag}_bicgstab"] = (("convdiff3d", 96, pe), "bicgstab", "xstar11",
                                     dict(SYN, maxIter=5000, relTol=1e-8, **JAC23))
        C[f"cd96_{tag}_gmres"] = (("convdiff3d", 96, pe), "gmres", "xstar11",
                                  dict(SYN, maxIter=5000, relTol=1e-8, **JAC23, **GM30))
        C[f"cd96_{tag}_fgmres300"] = (("convdiff3d", 96, pe), "fgmres", "xstar11",
                                      dict(SYN, maxIter=300, relTol=1e-8, **JAC23, **GM30))
        # the reference's default variable restart (between 10 and 30, GMRES.cxx:255-265)
        C[f"cd96_{tag}_gmresvar"] = (("convdiff3d", 96, pe), "gmres", "xstar11",
                                     dict(SYN, maxIter=5000, relTol=1e-8, **JAC23))
    return C


def build_matrix(spec):
    from faspxx_b200 import problems as P
    if spec[0] == "poisson2d":
        return P.poisson2d(spec[1])
    if spec[0] == "poisson3d":
        return P.poisson3d(spec[1])
    if spec[0] == "convdiff3d":
        return P.convdiff3d(spec[1], spec[2])
    raise KeyError(spec)


def rhs(A, kind):
    from faspxx_b200 import problems as P
    if kind == "xstar01":
        return A.matvec(P.seeded_uniform(A.nrow, 42))
    if kind == "xstar11":
        return A.matvec(P.seeded_uniform(A.nrow, 42, -1.0, 1.0))
    raise KeyError(kind)


def sample_index(n: int, seed: int = 2024) -> np.ndarray:
    k = min(NSAMPLE, n)
    return np.sort(np.random.default_rng(seed).choice(n, size=k, replace=False)).astype(np.int64)


def vardiff64():
    """The differentiable workload's inputs (64^3, kappa = exp(N(0,1)), b, x_t ~ N(0,1))."""
    from faspxx_b200 import problems as P
    rng = np.random.default_rng(42)
    N = 64
    kappa = np.exp(rng.standard_normal(N ** 3))
    A = P.vardiff3d(N, kappa)
    b = rng.standard_normal(A.nrow)
    xt = rng.standard_normal(A.nrow)
    return A, b, xt


def directions(n: int, nnz: int, count: int = 32, seed: int = 7):
    """Seeded directions (in b and in A's values) for the gradient projections."""
    rng = np.random.default_rng(seed)
    return [(rng.standard_normal(n), rng.standard_normal(nnz)) for _ in range(count)]


def _same(a, b) -> bool:
    return a.code == b.code and a.iters == b.iters and \
        np.array_equal(a.x.view(np.uint64), b.x.view(np.uint64)) and \
        a.norm2 == b.norm2


def run_solver_case(name: str):
    from oracle import oracle as O
    spec, alg, rk, kw = solver_cases()[name]
    A = build_matrix(spec)
    b = rhs(A, rk)
    x0 = np.zeros(A.nrow)
    t0 = time.perf_counter()
    ref = O.Solver("ref", A, alg, **kw).solve(b, x0)
    t_ref = time.perf_counter() - t0
    port = O.Solver("port", A, alg, **kw).solve(b, x0)
    if not _same(ref, port):
        raise AssertionError(f"{name}: restatement differs from the reference")
    # the reference prints its history with 6 significant digits
    m = min(len(ref.hist), len(port.hist))
    fin = np.isfinite(ref.hist[:m])
    rel = np.abs(ref.hist[:m][fin] - port.hist[:m][fin]) / np.maximum(port.hist[:m][fin], 1e-300)
    if rel.size and rel.max() > 1e-5:
        raise AssertionError(f"{name}: printed history differs ({rel.max():.2e})")
    idx = sample_index(A.nrow)
    # sensitivity envelope: every entry of b moved by one ulp, up or down, four seeded
    # times; per entry the largest deviation of the four histories, the iteration counts and
    # the largest solution difference
    env = np.zeros(len(port.hist))
    its, xdev, codes = [], 0.0, []
    for seed in ENV_SEEDS:
        up = np.random.default_rng(seed).random(A.nrow) < 0.5
        bp = np.where(up, np.nextafter(b, np.inf), np.nextafter(b, -np.inf))
        pert = O.Solver("port", A, alg, **kw).solve(bp, x0)
        mp = min(len(pert.hist), len(port.hist))
        dev = np.abs(pert.hist[:mp] - port.hist[:mp]) / np.maximum(port.hist[:mp], 1e-300)
        env[:mp] = np.fmax(env[:mp], dev)
        if mp < len(env):
            env[mp:] = np.inf  # a perturbed run stopped earlier: nothing to compare
        its.append(pert.iters)
        codes.append(pert.code)
        xdev = max(xdev, float(np.max(np.abs(pert.x[idx] - ref.x[idx])) / np.max(np.abs(ref.x))))
    over = np.nonzero(env > 1e-10)[0]
    envelope = dict(iters=its, codes=codes, hist_max=float(np.nanmax(env[np.isfinite(env)])),
                    first_over_1e10=int(over[0]) if len(over) else None, x_dev=xdev,
                    seeds=list(ENV_SEEDS))
    meta = dict(alg=alg, spec=list(spec), rhs=rk, kw=kw, n=A.nrow, nnz=A.nnz, code=ref.code,
                iters=ref.iters, norm2=ref.norm2, normInf=ref.normInf,
                x_norm2=float(np.linalg.norm(ref.x)), x_sum=float(ref.x.sum()),
                x_maxabs=float(np.max(np.abs(ref.x))),
                true_rel_residual=float(np.linalg.norm(b - A.matvec(ref.x)) / np.linalg.norm(b)),
                ref_seconds=round(t_ref, 2), restatement_bit_identical=True,
                envelope=envelope)
    arr = {"hist": port.hist, "hist_printed": ref.hist, "x_idx": idx, "x_val": ref.x[idx],
           "env_dev": env}
    return name, meta, arr


def run_adjoint():
    from oracle import oracle as O
    A, b, xt = vardiff64()
    n, nnz = A.nrow, A.nnz
    kw = dict(SYN, maxIter=20000, relTol=1e-10, **JAC1)
    fwd = O.Solver("ref", A, "cg", **kw).solve(b, np.zeros(n))
    fwd_p = O.Solver("port", A, "cg", **kw).solve(b, np.zeros(n))
    if not _same(fwd, fwd_p):
        raise AssertionError("vd64 forward: restatement differs from the reference")
    trp, tci, tva, _ = O.transpose("ref", A)
    from faspxx_b200 import problems as P
    AT = P.CSRMatrix(A.mcol, A.nrow, trp, tci, tva)
    g = fwd.x - xt
    adj = O.Solver("ref", AT, "cg", **kw).solve(g, np.zeros(n))
    adj_p = O.Solver("port", AT, "cg", **kw).solve(g, np.zeros(n))
    if not _same(adj, adj_p):
        raise AssertionError("vd64 adjoint: restatement differs from the reference")
    lam, x = adj.x, fwd.x
    rows = np.repeat(np.arange(n), np.diff(A.rowPtr.astype(np.int64)))
    gA = -lam[rows] * x[A.colInd.astype(np.int64)]
    proj = np.array([float(np.dot(lam, db) + np.dot(gA, da)) for db, da in directions(n, nnz)])
    ib, iA = sample_index(n), sample_index(nnz, 2025)
    meta = dict(n=n, nnz=nnz, forward_iters=fwd.iters, forward_code=fwd.code,
                adjoint_iters=adj.iters, adjoint_code=adj.code,
                grad_b_norm2=float(np.linalg.norm(lam)), grad_A_norm2=float(np.linalg.norm(gA)),
                loss=float(0.5 * np.dot(g, g)), kw=kw, restatement_bit_identical=True,
                directions="32 seeded (default_rng(7)) standard-normal pairs (db, dA values)")
    arr = {"proj": proj, "b_idx": ib, "b_val": lam[ib], "A_idx": iA, "A_val": gA[iA],
           "x_idx": ib, "x_val": x[ib], "fwd_hist": fwd_p.hist, "adj_hist": adj_p.hist}
    return "vd64_adjoint", meta, arr


def batch_sample(count: int = 4096, per_bin: int = 8):
    """A stratified sample of the batch: ``per_bin`` systems from each of 8 bins of m."""
    from faspxx_b200 import problems as P
    ms, sig, rhs_ = P.batch_systems(count=count, nrhs=4, seed=42)
    edges = np.linspace(16, 129, 9)
    rng = np.random.default_rng(3)
    pick = []
    for lo, hi in zip(edges[:-1], edges[1:]):
        cand = np.nonzero((ms >= lo) & (ms < hi))[0]
        pick.extend(sorted(rng.choice(cand, size=min(per_bin, len(cand)), replace=False)))
    return np.array(pick, np.int64), ms, sig, rhs_


def run_batch():
    from faspxx_b200 import problems as P
    from oracle import oracle as O
    pick, ms, sig, rhs_ = batch_sample()
    iters = np.zeros((len(pick), 4), np.int64)
    codes = np.zeros((len(pick), 4), np.int64)
    xs_idx, xs_val = [], []
    kw = dict(SYN, maxIter=5000, relTol=1e-8, **JAC1)
    for s, k in enumerate(pick):
        m = P.poisson2d(int(ms[k]), shift=float(sig[k]))
        idx = np.sort(np.random.default_rng(int(k)).choice(m.nrow, size=16, replace=False))
        solver = O.Solver("ref", m, "cg", **kw)
        port = O.Solver("port", m, "cg", **kw)
        for j in range(4):
            r = solver.solve(rhs_[k][j], np.zeros(m.nrow))
            if not _same(r, port.solve(rhs_[k][j], np.zeros(m.nrow))):
                raise AssertionError(f"batch system {k}: restatement differs")
            iters[s, j], codes[s, j] = r.iters, r.code
            xs_idx.append(idx)
            xs_val.append(r.x[idx])
    meta = dict(count=4096, sample=len(pick), kw=kw,
                stratification="8 equal-width bins of m over [16, 128], 8 systems each "
                               "(default_rng(3))")
    arr = {"systems": pick, "iters": iters, "codes": codes,
           "x_idx": np.stack(xs_idx), "x_val": np.stack(xs_val)}
    return "batch4096", meta, arr


def _job(name):
    if name == "vd64_adjoint":
        return run_adjoint()
    if name == "batch4096":
        return run_batch()
    return run_solver_case(name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--jobs", type=int, default=max(1, min(8, os.cpu_count() or 1)))
    a = ap.parse_args()
    from oracle import oracle as O
    if not os.path.exists(O.REF_SO):
        sys.exit("oracle/_ref/liboracle_ref.so is not built (make -C oracle)")
    names = list(solver_cases()) + ["vd64_adjoint", "batch4096"]
    if a.only:
        names = [n for n in names if n in a.only]
    jpath, npath = os.path.join(HERE, "fullsize.json"), os.path.join(HERE, "fullsize.npz")
    meta = json.load(open(jpath)) if os.path.exists(jpath) else {}
    arrs = dict(np.load(npath)) if os.path.exists(npath) else {}
    ctx = mp.get_context("spawn")
    with ctx.Pool(a.jobs) as pool:
        for name, m, arr in pool.imap_unordered(_job, names):
            meta[name] = m
            for k in [k for k in arrs if k.startswith(name + "__")]:
                del arrs[k]
            for k, v in arr.items():
                arrs[f"{name}__{k}"] = v
            print(name, {k: m[k] for k in m if k in ("code", "iters", "forward_iters",
                                                      "adjoint_iters", "ref_seconds")},
                  flush=True)
    with open(jpath, "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    np.savez_compressed(npath, **arrs)


if __name__ == "__main__":
    main()
