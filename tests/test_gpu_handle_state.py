"""mfgpu_analyze with the reference's own symbolic arrays, and the state a
rejected call leaves behind.

The Julia host hands libmfgpu the SymbolicMF it computed itself
(src/symbolic.jl:203-209: qf, parent, sstart and the update sets); the
factorization from those arrays must equal the oracle's.  An inconsistent
set is rejected on the host before any map reaches the device, and the
handle is then unanalyzed: factor and solve report a call-order error
instead of running the previous analysis's device maps against a
half-built plan.  A single-system analysis also ends a batch analysis.  A
factor call rejected for its arguments leaves the previous factorization
in place.
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


def test_rejected_factor_call_keeps_the_factorization():
    A = M.poisson3d(8)
    ctx = GpuContext()
    ctx.analyze(A, symbolic_mf(A))
    assert ctx.factor(A.nzval, None, False) == 0
    b = M.rhs(A.n, seed=2)
    x0 = ctx.solve(b, 0)
    assert ctx._lib.mfgpu_factor(ctx._h, None, None, 0) == -1
    assert ctx._lib.mfgpu_factor_scaled(ctx._h, None, 1, 0) == -1
    assert ctx._lib.mfgpu_factor_device(ctx._h, None, None, 0) == -1
    assert ctx._lib.mfgpu_factor_f32(ctx._h, None, None, 0) == -1
    np.testing.assert_array_equal(ctx.solve(b, 0), x0)


def test_device_entry_points_check_pointers_and_leading_dimensions():
    import ctypes

    import torch

    A = M.poisson3d(8)
    n, k = A.n, 2
    ctx = GpuContext()
    ctx.analyze(A, symbolic_mf(A))
    assert ctx.factor(A.nzval, None, False) == 0
    B = M.rhs(n, seed=4, nrhs=k)
    d_b = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).cuda()
    d_x = torch.zeros_like(d_b)
    out = ctypes.c_double()
    lib, h = ctx._lib, ctx._h
    null = ctypes.c_void_p(None)
    # rejected on the host before any launch (the buffers hold n * k values,
    # so even the short leading dimension would read in bounds)
    assert lib.mfgpu_solve_device(h, k, null, n, d_x.data_ptr(), n, 0) == -1
    assert lib.mfgpu_solve_device(h, k, d_b.data_ptr(), n, null, n, 0) == -1
    assert lib.mfgpu_solve_device(h, k, d_b.data_ptr(), n - 1, d_x.data_ptr(), n, 0) == -1
    assert lib.mfgpu_backward_error_device(h, k, null, n, d_x.data_ptr(), n, ctypes.byref(out)) == -1
    assert lib.mfgpu_backward_error_device(h, k, d_b.data_ptr(), n, d_x.data_ptr(), n - 1, ctypes.byref(out)) == -1
    # the handle still solves, and the backward error of that solve is tiny
    assert lib.mfgpu_solve_device(h, k, d_b.data_ptr(), n, d_x.data_ptr(), n, 0) == 0
    torch.cuda.synchronize()
    assert lib.mfgpu_backward_error_device(h, k, d_b.data_ptr(), n, d_x.data_ptr(), n, ctypes.byref(out)) == 0
    assert out.value <= 1e-14


def test_empty_matrix():
    # a 0 x 0 matrix: empty factors and solutions, as the oracle gives them
    from helpers import assert_same_structure
    from pureumfpack import SparseCSC, multifrontal_lu, splu

    A = SparseCSC(0, 0, np.array([1]), np.zeros(0, np.int64), np.zeros(0))
    x = splu(A, method="multifrontal").ldiv(np.zeros(0))
    assert x.shape == (0,)
    G = multifrontal_lu(A)
    fo = O.multifrontal_lu(A)
    assert_same_structure(fo, G.L, G.U, G.p, G.q, G.pinv)
