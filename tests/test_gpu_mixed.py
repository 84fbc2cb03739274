"""The mixed-precision form against the oracle's FP64 factorization.

FP32 fronts give the reference's structure exactly (fill, row order, and the
same pivot sequence on these diagonally dominant and mildly unsymmetric
matrices) with factor values to FP32 accuracy; FP64 refinement through
solve(F, b; refine) (src/interface.jl:170-177) then brings the normwise
backward error to the FP64 level.  The Schur updates run on tcgen05 tensor
cores as 3xTF32 split products by default, or as SIMT FP32 (the tensor-core
switch off); both must meet the same bounds.
"""

import numpy as np
import pytest

from helpers import column_value_errors
from oracle import oracle as O
from pureumfpack import PRECISION_MIXED, SCALE_SUM, GpuContext, row_scaling, solve, splu, symbolic_mf
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu

# normwise per-column agreement of FP32-front factors with the FP64 oracle
MIXED_RTOL = 2e-5
TARGET_ETA = 1e-14


def _eta(A, x, b):
    S = A.to_scipy()
    x = x.reshape(A.n, -1)
    b = b.reshape(A.n, -1)
    r = b - S @ x
    anorm = np.max(np.asarray(abs(S).sum(axis=1)).ravel())
    return float(np.max(np.abs(r).max(axis=0) / (anorm * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))))


def _mixed_factors(A, tensor_cores, tf32_split=False):
    S = symbolic_mf(A)
    Rs = row_scaling(A, SCALE_SUM)
    ctx = GpuContext(precision=PRECISION_MIXED, tensor_cores=tensor_cores, tf32_split=tf32_split)
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, Rs, True) == 0
    return ctx.factors()


CASES = [("poisson3d-20", lambda: M.poisson3d(20)), ("convdiff-14", lambda: M.convdiff3d(14)),
         ("poisson2d-100", lambda: M.poisson2d(100))]


@pytest.mark.parametrize("tensor_cores,tf32_split", [(True, False), (True, True), (False, False)],
                         ids=["bf16x3", "3xtf32", "simt"])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_mixed_factors_match_fp64_oracle(name, make, tensor_cores, tf32_split):
    A = make()
    fo = O.splu(A, scale=int(SCALE_SUM)).F
    L, U, p, q, pinv = _mixed_factors(A, tensor_cores, tf32_split)
    np.testing.assert_array_equal(L.colptr, fo.Lcolptr)
    np.testing.assert_array_equal(L.rowval, fo.Lrowval)
    np.testing.assert_array_equal(U.rowval, fo.Urowval)
    np.testing.assert_array_equal(p, fo.p)
    nl, _ = column_value_errors(fo.Lcolptr, fo.Lnzval, L.nzval)
    nu, _ = column_value_errors(fo.Ucolptr, fo.Unzval, U.nzval)
    assert nl <= MIXED_RTOL and nu <= MIXED_RTOL, (nl, nu)


@pytest.mark.parametrize("tf32_split", [False, True], ids=["bf16x3", "3xtf32"])
def test_tensor_core_and_simt_updates_agree(tf32_split):
    A = M.poisson3d(22)
    Lt, Ut = _mixed_factors(A, True, tf32_split)[:2]
    Ls, Us = _mixed_factors(A, False)[:2]
    nl, _ = column_value_errors(Ls.colptr, Ls.nzval, Lt.nzval)
    nu, _ = column_value_errors(Us.colptr, Us.nzval, Ut.nzval)
    assert nl <= MIXED_RTOL and nu <= MIXED_RTOL, (nl, nu)


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_mixed_refinement_reaches_fp64_backward_error(name, make):
    A = make()
    B = M.rhs(A.n, seed=4, nrhs=8)
    F = splu(A, method="multifrontal", precision=PRECISION_MIXED)
    x0 = solve(F, B, refine=0)
    assert _eta(A, x0, B) <= 1e-6           # FP32 factors alone
    x = solve(F, B, refine=3)
    assert _eta(A, x, B) <= TARGET_ETA
    xo = O.solve(O.splu(A), B, refine=1)
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)


def test_growth_check_refactors_in_fp64():
    """Mixed form: element growth above the limit sends the matrix back to an
    FP64 factorization; the factors are then exactly the FP64 form's."""
    A = M.convdiff3d(10)
    S = symbolic_mf(A)
    Rs = row_scaling(A, SCALE_SUM)
    ref = GpuContext(precision=0)
    ref.analyze(A, S)
    assert ref.factor(A.nzval, Rs, True) == 0
    L0, U0 = ref.factors()[:2]

    ctx = GpuContext(precision=PRECISION_MIXED)
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, Rs, True) == 0
    st = ctx.stats()
    assert st["refactored_fp64"] is False and 0 < st["growth"] < st["growth_limit"]
    assert st["precision"] == "mixed"

    ctx.set_growth_limit(1e-30)               # any growth now exceeds the limit
    assert ctx.factor(A.nzval, Rs, True) == 0
    st = ctx.stats()
    assert st["refactored_fp64"] is True and st["precision"] == "fp64"
    L1, U1 = ctx.factors()[:2]
    np.testing.assert_array_equal(L1.nzval, L0.nzval)
    np.testing.assert_array_equal(U1.nzval, U0.nzval)
    B = M.rhs(A.n, seed=1, nrhs=3)
    assert _eta(A, ctx.solve(B, 0), B) <= 1e-14
