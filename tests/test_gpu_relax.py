"""Relaxed amalgamation on the GPU (opt-in): the factors of the coarser
supernodal structure reconstruct Rs .* A to the reference tests' bound
(test/multifrontal_test.jl:38-39) and solve to the oracle's solution; the
entries the merges add are explicit zeros."""

import numpy as np
import pytest

from helpers import reconstruction_error
from oracle import oracle as O
from pureumfpack import PRECISION_MIXED, solve, splu
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,make", [("poisson3d-18", lambda: M.poisson3d(18)),
                                       ("convdiff-12", lambda: M.convdiff3d(12)),
                                       ("poisson2d-80", lambda: M.poisson2d(80))])
def test_relaxed_factorization(name, make):
    A = make()
    F0 = splu(A, method="multifrontal")
    F = splu(A, method="multifrontal", relax=True)
    assert reconstruction_error(A, F.L, F.U, F.p, F.q, Rs=F.Rs) <= 1e-9
    assert len(F.L.nzval) >= len(F0.L.nzval)
    B = M.rhs(A.n, seed=5, nrhs=3)
    x = solve(F, B, refine=1)
    xo = O.solve(O.splu(A), B, refine=1)
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)


def test_relaxed_mixed_precision_reaches_fp64_accuracy():
    A = M.poisson3d(16)
    B = M.rhs(A.n, seed=5, nrhs=4)
    F = splu(A, method="multifrontal", relax=True, precision=PRECISION_MIXED)
    x = solve(F, B, refine=3)
    S = A.to_scipy()
    r = B - S @ x
    eta = np.max(np.abs(r).max(0) / (np.abs(S).sum(1).max() * np.abs(x).max(0) + np.abs(B).max(0)))
    assert eta <= 1e-14
