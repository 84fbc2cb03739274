"""Bounded device waits: a wait that runs out is a status, not a hang.

The tensor-core GEMMs of the FP32 fronts (register-staged and bulk-copy
forms) synchronise their warps through mbarriers, and the persistent solve
synchronises its CTAs through a grid barrier; every one of these waits is
bounded by the handle's wait limit
(mfgpu_set_wait_limit, 4 s by default).  The test hook mfgpu_test_stall makes
a wait that can never complete -- the GEMMs' MMA issuer waits on an mbarrier
that nothing arrives at, CTA 0 of the persistent solve never arrives at its
grid barrier -- so the waits run out by the kernels' own clocks.  The calls
must then return MFGPU_ERR_TIMEOUT (no trap, no fault), a factorization that
gave up must leave no factors, and the same handle must factor and solve
normally once the hook is off, bit for bit as before -- which also shows that
the kernels that gave up freed their tensor memory (a later allocation of it
would otherwise wait for ever).  The reference reports failures as a status
too (src/multifrontal.jl:250-252).
"""

import time

import numpy as np
import pytest

from helpers import backward_error
from pureumfpack import PRECISION_FP64, PRECISION_MIXED, GpuContext, MfgpuError, row_scaling, symbolic_mf
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu

MFGPU_ERR_TIMEOUT = -5
MFGPU_ERR_STATE = -4


@pytest.mark.parametrize("k", [20, 40], ids=["poisson3d-20", "poisson3d-40"])
def test_tensor_core_wait_runs_out_and_the_handle_recovers(k):
    # poisson3d-40 has long-K Schur updates, so the bulk-copy GEMM
    # (k_gemm_bx3p) gives up its waits too: its producer lets the copies in
    # flight land before the CTA ends
    A = M.poisson3d(k)
    S = symbolic_mf(A)
    Rs = row_scaling(A, 1)
    b = M.rhs(A.n, seed=6)
    ctx = GpuContext(device=0, precision=PRECISION_MIXED)
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, Rs, True) == 0
    x_ref = ctx.solve(b, refine=2)

    ctx.set_wait_limit(1e-4)
    ctx.test_stall(True)
    t0 = time.perf_counter()
    with pytest.raises(MfgpuError) as e:
        ctx.factor(A.nzval, Rs, True)
    assert e.value.code == MFGPU_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 60.0
    # no factors survive a factorization that gave up
    with pytest.raises(MfgpuError) as e:
        ctx.solve(b)
    assert e.value.code == MFGPU_ERR_STATE

    ctx.test_stall(False)
    ctx.set_wait_limit(4.0)
    assert ctx.factor(A.nzval, Rs, True) == 0
    x = ctx.solve(b, refine=2)
    assert backward_error(A, x, b) <= 1e-14
    np.testing.assert_array_equal(x, x_ref)   # same launches, same arithmetic: bitwise the first solve


def test_persistent_solve_barrier_runs_out_and_the_handle_recovers():
    A = M.poisson3d(12)
    S = symbolic_mf(A)
    Rs = row_scaling(A, 1)
    b = M.rhs(A.n, seed=8)
    ctx = GpuContext(device=0, precision=PRECISION_FP64, persistent_solve=True)
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, Rs, True) == 0
    x_ref = ctx.solve(b, refine=1)

    ctx.set_wait_limit(1e-3)
    ctx.test_stall(True)
    with pytest.raises(MfgpuError) as e:
        ctx.solve(b, refine=1)
    assert e.value.code == MFGPU_ERR_TIMEOUT

    ctx.test_stall(False)
    ctx.set_wait_limit(4.0)
    x = ctx.solve(b, refine=1)   # the factors are intact: only the solve gave up
    np.testing.assert_array_equal(x, x_ref)
    assert backward_error(A, x, b) <= 1e-14


def test_wait_limit_is_checked():
    ctx = GpuContext(device=0)
    for bad in (0.0, -1.0, float("nan"), 1e9):
        with pytest.raises(Exception):
            ctx.set_wait_limit(bad)
