"""The backward-error entry point that allocates no device memory.

mfgpu_backward_error_noalloc serves callers that cannot allocate device
memory when they check accuracy (services that reserve all device memory at
start-up, loops that must not take cudaMalloc's device-wide
synchronisation).  It must give the same normwise backward error as
mfgpu_backward_error_device, call after call, although every call reuses
the same fixed device array.  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

from pureumfpack import matrices as M
from pureumfpack import splu

pytestmark = pytest.mark.gpu


def _eta(ctx, fn, nrhs, b, x, n):
    out = ctypes.c_double()
    rc = fn(ctx._h, nrhs, ctypes.c_void_p(b.data_ptr()), n, ctypes.c_void_p(x.data_ptr()), n, ctypes.byref(out))
    assert rc == 0, ctx._lib.mfgpu_last_error(ctx._h).decode()
    return out.value


def test_noalloc_matches_allocating_entry_point():
    import torch

    A = M.poisson3d(12)
    n, nrhs = A.n, 5
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    lib = ctx._lib
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
        ref = _eta(ctx, lib.mfgpu_backward_error_device, nrhs, d_b, x, n)
        got = _eta(ctx, lib.mfgpu_backward_error_noalloc, nrhs, d_b, x, n)
        assert got == pytest.approx(ref, rel=1e-12, abs=0.0)
        results.append(got)
    assert results[0] <= 1e-14
    assert results[1] > 100 * results[0]
    assert results[2] == results[0]


def test_noalloc_rejects_too_many_rhs():
    A = M.poisson2d(6)
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    out = ctypes.c_double()
    rc = ctx._lib.mfgpu_backward_error_noalloc(ctx._h, 4097, ctypes.c_void_p(8), A.n, ctypes.c_void_p(8), A.n,
                                               ctypes.byref(out))
    assert rc == -1
    assert b"4096" in ctx._lib.mfgpu_last_error(ctx._h)
