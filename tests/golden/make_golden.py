"""Generate the golden fixtures under tests/golden/ from the FASP++ reference itself.

Run in a container that has the reference tree (default /root/reference) after
``make -C oracle``; the GPU box never runs this script, it only reads its outputs:

* ``fdm_10X10.npz``, ``fem_small.npz`` -- the reference's bundled matrices
  (data/fdm_10X10.csr, data/fem_small.csr) as 0-based uint32/float64 CSR arrays;
* ``known_answers.json`` -- the small known-answer cases of the reference's unit tests
  (utest/src/UnitTestsMAT.cxx:42-67,152-161; utest/src/UnitTestsJacobi.cxx:23-157;
  example/TestWeightedJacobi.cxx:60-136);
* ``reference_runs.npz`` + ``reference_runs.json`` -- outputs of the compiled reference
  (oracle/_ref/liboracle_ref.so) for every solver configuration the tests replay: return
  code, iteration count, norms, the solution x and the printed residual history;
* ``reference_transpose.npz`` -- MAT::TransInPlace results, the bit-exact target for CSC.

    python tests/golden/make_golden.py [/path/to/reference]
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from faspxx_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden import cases as G  # noqa: E402


def check_against_readmat(path: str, A: P.CSRMatrix) -> None:
    """The Python reader must give exactly the MAT the reference's ReadMat builds."""
    lib = O.load("ref")
    nrow, nnz = C.c_uint32(), C.c_uint32()
    lib.orc_ref_readmat.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                    C.c_void_p, C.c_void_p, C.c_void_p]
    assert lib.orc_ref_readmat(path.encode(), C.byref(nrow), C.byref(nnz), None, None, None) == 0
    rp = np.empty(nrow.value + 1, np.uint32)
    ci = np.empty(nnz.value, np.uint32)
    va = np.empty(nnz.value, np.float64)
    lib.orc_ref_readmat(path.encode(), C.byref(nrow), C.byref(nnz), rp.ctypes.data,
                        ci.ctypes.data, va.ctypes.data)
    assert np.array_equal(rp, A.rowPtr) and np.array_equal(ci, A.colInd)
    assert np.array_equal(va, A.values)


def main(ref_root: str) -> None:
    O.build(ref=True)
    mats = {}
    for name in ("fdm_10X10", "fem_small"):
        path = os.path.join(ref_root, "data", name + ".csr")
        A = P.read_csr_text(path)
        check_against_readmat(path, A)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), rowPtr=A.rowPtr,
                            colInd=A.colInd, values=A.values)
        mats[name] = A

    runs_meta, runs_arr = {}, {}
    for case in G.solver_cases():
        A, b, x0 = G.case_inputs(case)
        s = O.Solver("ref", A, case["alg"], **case["kw"])
        outs = []
        for rep in range(case.get("repeat", 1)):
            r = s.solve(b, x0)
            outs.append(r)
        for rep, r in enumerate(outs):
            key = case["name"] if rep == 0 else f"{case['name']}__rep{rep}"
            runs_meta[key] = dict(code=r.code, iters=r.iters, norm2=r.norm2, normInf=r.normInf)
            runs_arr[key + "__x"] = r.x
            runs_arr[key + "__hist"] = r.hist
        if case.get("store_b"):
            runs_arr[case["name"] + "__b"] = b
    np.savez_compressed(os.path.join(HERE, "reference_runs.npz"), **runs_arr)
    with open(os.path.join(HERE, "reference_runs.json"), "w") as f:
        json.dump(runs_meta, f, indent=1, sort_keys=True)

    tr = {}
    for name, A in G.transpose_cases():
        rp, ci, va, dp = O.transpose("ref", A)
        tr[name + "__rowPtr"], tr[name + "__colInd"], tr[name + "__diagPtr"] = rp, ci, dp
        if va is not None:
            tr[name + "__values"] = va
    np.savez_compressed(os.path.join(HERE, "reference_transpose.npz"), **tr)
    print("wrote", len(runs_meta), "solver runs and", len(G.transpose_cases()), "transposes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
