"""The reference's matrix-free example (example/TestMatFree.cxx) on the CPU oracle.

Its operator (MatFree::Apply, :97-176) is the 5-point Laplacian on the (dim-1)^2 interior
grid with the entries summed in ascending column order, so CG on the assembled matrix
repeats the example's arithmetic: the oracle, given the example's right-hand side
(orc_matfree_rhs) and start (x = 0.25), must print what the reference printed
(tests/golden/reference_matfree.json): the same iteration counts and the same norms and
L2 errors to the 5 digits shown.
"""
import json
import os

import numpy as np
import pytest

from faspxx_b200 import problems as P

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                   "reference_matfree.json")))


def l2_error(dim, x):
    """The example's error: sqrt(h^2 sum (x - sin(pi x) sin(pi y))^2) (TestMatFree.cxx:236-243)."""
    h = 1.0 / dim
    k = np.arange(1, dim)
    u = np.outer(np.sin(np.pi * k * h), np.sin(np.pi * k * h)).ravel()
    return float(np.sqrt(np.sum((x - u) ** 2) * h * h))


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    oracle.build(ref=False)
    return oracle


@pytest.mark.parametrize("dim", [16, 32, 64, 128])
def test_oracle_repeats_the_matrix_free_example(O, dim):
    ref = GOLD[str(dim)]
    A = P.poisson2d(dim - 1)
    b = O.matfree_rhs(dim)
    r = O.solve("port", A, "cg", b, np.full(A.nrow, 0.25), maxIter=10000, restart=20,
                relTol=1e-8, absTol=1e-12)
    assert r.iters == ref["iters"]
    assert f"{r.norm2:.4e}" == ref["norm2"]
    assert f"{r.normInf:.4e}" == ref["normInf"]
    assert f"{l2_error(dim, r.x):.4e}" == ref["l2err"]
