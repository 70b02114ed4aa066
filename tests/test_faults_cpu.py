"""Bad inputs on the host side: the C restatement against the reference itself (both run
here on the CPU) on NaN/Inf in b, NaN in x0, a zero diagonal under Jacobi, maxIter = 1,
b = x0 = 0 and a zero matrix, for CG, BiCGStab, GMRES and FGMRES with and without a Jacobi
preconditioner (tests/golden/cases.py: fault_cases). The same return code, iteration
count and residual norm (NaN where the reference's is NaN), and the same solution bit for
bit where the reference defines it. The GPU is held to these outcomes in
tests/test_gpu_faults.py."""
import os

import numpy as np
import pytest

from tests.golden import cases as G

CASES = G.fault_cases()


@pytest.fixture(scope="module")
def oracle():
    from oracle import oracle as O
    O.build(ref=False)
    if not os.path.exists(O.REF_SO):
        pytest.skip("the reference is not built here")
    return O


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference_on_faults(oracle, name):
    alg, kw, A, b, x0, cmpx = CASES[name]
    ref = oracle.Solver("ref", A, alg, **kw).solve(b, x0)
    port = oracle.Solver("port", A, alg, **kw).solve(b, x0)
    assert (port.code, port.iters) == (ref.code, ref.iters), name
    assert np.isnan(port.norm2) == np.isnan(ref.norm2), name
    if not np.isnan(ref.norm2):
        assert port.norm2 == ref.norm2, name
    if cmpx:
        assert np.array_equal(port.x, ref.x, equal_nan=True), name
