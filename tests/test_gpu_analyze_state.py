"""mfgpu_analyze with the reference's own symbolic arrays, and the state a
failed analysis leaves behind.

The Julia host hands libmfgpu the SymbolicMF it computed itself
(src/symbolic.jl:203-209: qf, parent, sstart and the update sets); the
factorization from those arrays must equal the oracle's.  An inconsistent
set is rejected on the host before any map reaches the device, and the
handle is then unanalyzed: factor and solve report a call-order error
instead of running the previous analysis's device maps against a
half-built plan.  A single-system analysis also ends a batch analysis.
None of these cases hands a kernel an inconsistent map: the rejections
happen in host code before the first upload.
"""

import numpy as np
import pytest

from helpers import assert_close_values, assert_same_structure
from oracle import oracle as O
from pureumfpack import ArgumentError, GpuContext, colamd_order, splu_batch, symbolic_mf
from pureumfpack import matrices as M
from pureumfpack.api import GPLUFactorization, MfgpuError, analyze_batch

pytestmark = pytest.mark.gpu

ERR_STATE = -4


@pytest.mark.parametrize("merge", [True, False])
def test_reference_symbolic_arrays_factor_like_the_oracle(merge):
    A = M.convdiff3d(10)
    q = colamd_order(A)
    S = symbolic_mf(A, q=q)
    ctx = GpuContext(merge_fronts=merge)
    ctx.analyze_arrays(A, S.qf, S.parent, S.sstart, S.upd_ptr, S.upd_idx)
    assert ctx.factor(A.nzval, None, False) == 0
    F = GPLUFactorization(ctx)
    fo = O.multifrontal_lu(A, q=q, check=False)
    assert_same_structure(fo, F.L, F.U, F.p, F.q, F.pinv)
    assert_close_values(fo, F.L, F.U)


def test_failed_analysis_leaves_the_handle_unanalyzed():
    A = M.poisson3d(8)
    S = symbolic_mf(A)
    ctx = GpuContext()
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, None, False) == 0
    b = M.rhs(A.n, seed=1)
    x0 = ctx.solve(b, 0)
    # a partition that stops one column short of n
    short = S.sstart.copy()
    short[-1] = A.n
    with pytest.raises(ArgumentError):
        ctx.analyze_arrays(A, S.qf, S.parent, short, S.upd_ptr, S.upd_idx)
    with pytest.raises(MfgpuError) as e:
        ctx.factor(A.nzval, None, False)
    assert e.value.code == ERR_STATE
    with pytest.raises(MfgpuError) as e:
        ctx.solve(b, 0)
    assert e.value.code == ERR_STATE
    # an update row outside the matrix
    bad = S.upd_idx.copy()
    bad[0] = A.n + 1
    with pytest.raises(ArgumentError):
        ctx.analyze_arrays(A, S.qf, S.parent, S.sstart, S.upd_ptr, bad)
    # the same handle analyzes and factors again
    ctx.analyze_arrays(A, S.qf, S.parent, S.sstart, S.upd_ptr, S.upd_idx)
    assert ctx.factor(A.nzval, None, False) == 0
    np.testing.assert_allclose(ctx.solve(b, 0), x0, rtol=1e-13, atol=0)


def test_single_system_analysis_ends_the_batch():
    As = [M.poisson3d(6), M.poisson2d(20)]
    ctx = analyze_batch(As)
    splu_batch(As, ctx=ctx)
    A = M.poisson3d(9)
    ctx.analyze(A, symbolic_mf(A))
    with pytest.raises(MfgpuError) as e:
        splu_batch(As, ctx=ctx, check=False)
    assert e.value.code == ERR_STATE
    assert ctx.factor(A.nzval, None, False) == 0
