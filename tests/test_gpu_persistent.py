"""The persistent solve (one cooperative launch per pass) against the
one-launch-per-step solve and the oracle.

Both run the same per-step item code over the same schedule, the persistent
one with bounded grid barriers between dependent steps; their solutions must
agree to rounding and match the oracle's solve(F, b; refine)
(src/interface.jl:170-177), in both precisions and for many and few
right-hand sides.
"""

import numpy as np
import pytest

from oracle import oracle as O
from pureumfpack import PRECISION_FP64, PRECISION_MIXED, GpuContext, row_scaling, symbolic_mf
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


def _solve(A, B, precision, persistent, refine):
    S = symbolic_mf(A)
    Rs = row_scaling(A, 1)
    ctx = GpuContext(precision=precision, persistent_solve=persistent)
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, Rs, True) == 0
    X = ctx.solve(B, refine)
    X2 = ctx.solve(B, refine)          # a second pass over the same schedule (graph replay)
    np.testing.assert_array_equal(X, X2)
    return X


@pytest.mark.parametrize("precision,refine", [(PRECISION_FP64, 0), (PRECISION_MIXED, 3)], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name,make,nrhs", [
    ("poisson3d-18", lambda: M.poisson3d(18), 70),
    ("convdiff-12", lambda: M.convdiff3d(12), 3),
    ("poisson2d-60", lambda: M.poisson2d(60), 1),
], ids=["poisson3d-18x70", "convdiff-12x3", "poisson2d-60x1"])
def test_persistent_solve_matches_step_launches(name, make, nrhs, precision, refine):
    A = make()
    B = M.rhs(A.n, seed=2, nrhs=nrhs)
    xp = _solve(A, B, precision, True, refine)
    xs = _solve(A, B, precision, False, refine)
    assert np.linalg.norm(xp - xs) <= 1e-12 * np.linalg.norm(xs)
    xo = O.solve(O.splu(A), B, refine=1)
    assert np.linalg.norm(xp - xo) <= 1e-10 * np.linalg.norm(xo)
