"""The backward-error entry point that allocates no device memory.

mfgpu_backward_error_noalloc serves callers that cannot allocate device
memory when they check accuracy (services that reserve all device memory at
start-up, loops that must not take cudaMalloc's device-wide
synchronisation).  It must give the same normwise backward error as
mfgpu_backward_error_device, call after call, although every call reuses
the same fixed device array: padded leading dimensions, the largest
right-hand-side count it accepts, Float32 and mixed-precision handles, a 0 x 0
system, and a NaN in the solution (both entry points must then report a
non-finite error).  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

from pureumfpack import PRECISION_MIXED, GpuContext, SparseCSC, row_scaling, splu, symbolic_mf
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu

MAX_RHS = 4096


def _eta(ctx, fn, nrhs, b, x, ldb, ldx):
    out = ctypes.c_double()
    rc = fn(ctx._h, nrhs, ctypes.c_void_p(b), ldb, ctypes.c_void_p(x), ldx, ctypes.byref(out))
    assert rc == 0, ctx._lib.mfgpu_last_error(ctx._h).decode()
    return out.value


def _both(ctx, nrhs, b, x, ldb, ldx):
    lib = ctx._lib
    ref = _eta(ctx, lib.mfgpu_backward_error_device, nrhs, b, x, ldb, ldx)
    got = _eta(ctx, lib.mfgpu_backward_error_noalloc, nrhs, b, x, ldb, ldx)
    return ref, got


def _padded(B, ld):
    """Device copy of B (n x nrhs) with leading dimension ld >= n."""
    import torch

    n, nrhs = B.shape
    P = np.full((ld, nrhs), 7.0)
    P[:n] = B
    return torch.from_numpy(P.ravel(order="F")).cuda()


def test_noalloc_matches_allocating_entry_point():
    import torch

    A = M.poisson3d(12)
    n, nrhs = A.n, 5
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    B = M.rhs(n, seed=7, nrhs=nrhs)
    d_b = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).cuda()
    d_x = torch.empty_like(d_b)
    ctx.solve_device(nrhs, d_b.data_ptr(), n, d_x.data_ptr(), n, 1)
    torch.cuda.synchronize()
    # a worse solution for the second call: the fixed array must not carry
    # over the first call's maxima
    d_x2 = d_x * (1.0 + 1e-6)
    results = []
    for x in (d_x, d_x2, d_x):
        ref, got = _both(ctx, nrhs, d_b.data_ptr(), x.data_ptr(), n, n)
        assert got == pytest.approx(ref, rel=1e-12, abs=0.0)
        results.append(got)
    assert results[0] <= 1e-14
    assert results[1] > 100 * results[0]
    assert results[2] == results[0]


def test_noalloc_padded_leading_dimensions():
    import torch

    A = M.convdiff3d(6)
    n, nrhs = A.n, 3
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    B = M.rhs(n, seed=11, nrhs=nrhs)
    ld = n + 3
    d_b = _padded(B, ld)
    d_x = torch.full((ld * nrhs,), 7.0, dtype=torch.float64, device="cuda")
    ctx.solve_device(nrhs, d_b.data_ptr(), ld, d_x.data_ptr(), ld, 1)
    torch.cuda.synchronize()
    for _ in range(2):
        ref, got = _both(ctx, nrhs, d_b.data_ptr(), d_x.data_ptr(), ld, ld)
        assert got == pytest.approx(ref, rel=1e-12, abs=0.0)
        assert got <= 1e-14
    # the padding rows (value 7) are not read: a solution written with
    # leading dimension ld gives the same error as its compact copy
    X = d_x.cpu().numpy().reshape(ld, nrhs, order="F")[:n]
    d_xc = torch.from_numpy(np.asfortranarray(X).ravel(order="F")).cuda()
    d_bc = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).cuda()
    ref_c, got_c = _both(ctx, nrhs, d_bc.data_ptr(), d_xc.data_ptr(), n, n)
    assert got_c == got


def test_noalloc_largest_rhs_count():
    import torch

    A = M.poisson2d(4)
    n = A.n
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    B = M.rhs(n, seed=3, nrhs=MAX_RHS)
    d_b = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).cuda()
    d_x = torch.empty_like(d_b)
    ctx.solve_device(MAX_RHS, d_b.data_ptr(), n, d_x.data_ptr(), n, 0)
    torch.cuda.synchronize()
    d_x[5 * n + 3] += 1e-3   # one column with a much larger error
    for _ in range(2):
        ref, got = _both(ctx, MAX_RHS, d_b.data_ptr(), d_x.data_ptr(), n, n)
        assert got == pytest.approx(ref, rel=1e-12, abs=0.0)
        assert got > 1e-6


@pytest.mark.parametrize("kind", ["float32", "mixed"])
def test_noalloc_float32_and_mixed_handles(kind):
    import torch

    A = M.poisson3d(8)
    n, nrhs = A.n, 4
    S = symbolic_mf(A)
    Rs = row_scaling(A, 1)
    if kind == "float32":
        ctx = GpuContext(device=0)
        ctx.analyze(A, S)
        ctx.factor_f32(A.nzval.astype(np.float32), Rs.astype(np.float32), True)
    else:
        ctx = GpuContext(device=0, precision=PRECISION_MIXED)
        ctx.analyze(A, S)
        ctx.factor(A.nzval, Rs, True)
    B = M.rhs(n, seed=5, nrhs=nrhs)
    d_b = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).cuda()
    d_x = torch.empty_like(d_b)
    ctx.solve_device(nrhs, d_b.data_ptr(), n, d_x.data_ptr(), n, 2)
    torch.cuda.synchronize()
    for _ in range(2):
        ref, got = _both(ctx, nrhs, d_b.data_ptr(), d_x.data_ptr(), n, n)
        assert got == pytest.approx(ref, rel=1e-12, abs=0.0)
        assert 0.0 < got <= 1e-10


def test_noalloc_nan_solution_is_not_finite():
    import torch

    A = M.poisson3d(6)
    n, nrhs = A.n, 3
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    B = M.rhs(n, seed=9, nrhs=nrhs)
    d_b = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).cuda()
    d_x = torch.empty_like(d_b)
    ctx.solve_device(nrhs, d_b.data_ptr(), n, d_x.data_ptr(), n, 0)
    torch.cuda.synchronize()
    good_ref, good = _both(ctx, nrhs, d_b.data_ptr(), d_x.data_ptr(), n, n)
    assert np.isfinite(good) and good <= 1e-14
    d_x[n + 17] = float("nan")   # one NaN entry in the second column
    ref, got = _both(ctx, nrhs, d_b.data_ptr(), d_x.data_ptr(), n, n)
    assert not np.isfinite(ref)
    assert not np.isfinite(got)
    d_x[n + 17] = float("inf")
    ref, got = _both(ctx, nrhs, d_b.data_ptr(), d_x.data_ptr(), n, n)
    assert not np.isfinite(ref) and not np.isfinite(got)
    # the next call with a finite solution is finite again: nothing sticks
    ctx.solve_device(nrhs, d_b.data_ptr(), n, d_x.data_ptr(), n, 0)
    torch.cuda.synchronize()
    ref, got = _both(ctx, nrhs, d_b.data_ptr(), d_x.data_ptr(), n, n)
    assert got == good and ref == good_ref


def test_noalloc_empty_system():
    A = SparseCSC(0, 0, np.array([1]), np.zeros(0, np.int64), np.zeros(0))
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    for fn in (ctx._lib.mfgpu_backward_error_device, ctx._lib.mfgpu_backward_error_noalloc):
        out = ctypes.c_double(-1.0)
        rc = fn(ctx._h, 1, None, 0, None, 0, ctypes.byref(out))
        assert rc == 0 and out.value == 0.0


def test_noalloc_rejects_too_many_rhs():
    A = M.poisson2d(6)
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    out = ctypes.c_double()
    rc = ctx._lib.mfgpu_backward_error_noalloc(ctx._h, MAX_RHS + 1, ctypes.c_void_p(8), A.n, ctypes.c_void_p(8),
                                               A.n, ctypes.byref(out))
    assert rc == -1
    assert b"4096" in ctx._lib.mfgpu_last_error(ctx._h)
