"""Bounded device waits: a wait that runs out is a status, not a hang.

The tensor-core GEMMs of the FP32 fronts synchronise their warps through
mbarriers, and every wait on them is bounded by the handle's wait limit
(mfgpu_set_wait_limit, 4 s by default).  Here the limit is cut to a
nanosecond, so the long-K Schur updates of poisson3d(32) run out of it: the
factorization must return MFGPU_ERR_TIMEOUT (no trap, no fault), leave no
factors behind, and the same handle must factor and solve normally once the
limit is restored -- which also shows that the kernels that gave up drained
their tensor-core work and freed their tensor memory (a later allocation of
it would otherwise wait for ever).  The reference reports failures as a
status too (src/multifrontal.jl:250-252).  No GPU fault is provoked: the
waits end by the kernels' own clocks.
"""

import time

import numpy as np
import pytest

from helpers import backward_error
from pureumfpack import PRECISION_MIXED, GpuContext, MfgpuError, row_scaling, symbolic_mf
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu

MFGPU_ERR_TIMEOUT = -5
MFGPU_ERR_STATE = -4


def test_tensor_core_wait_runs_out_and_the_handle_recovers():
    A = M.poisson3d(32)
    S = symbolic_mf(A)
    Rs = row_scaling(A, 1)
    b = M.rhs(A.n, seed=6)
    ctx = GpuContext(device=0, precision=PRECISION_MIXED)
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, Rs, True) == 0
    x_ref = ctx.solve(b, refine=2)

    ctx.set_wait_limit(1e-9)
    t0 = time.perf_counter()
    with pytest.raises(MfgpuError) as e:
        ctx.factor(A.nzval, Rs, True)
    assert e.value.code == MFGPU_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 60.0
    # no factors survive a factorization that gave up
    with pytest.raises(MfgpuError) as e:
        ctx.solve(b)
    assert e.value.code == MFGPU_ERR_STATE

    ctx.set_wait_limit(4.0)
    assert ctx.factor(A.nzval, Rs, True) == 0
    x = ctx.solve(b, refine=2)
    assert backward_error(A, x, b) <= 1e-14
    np.testing.assert_array_equal(x, x_ref)   # same launches, same arithmetic: bitwise the first solve


def test_wait_limit_is_checked():
    ctx = GpuContext(device=0)
    for bad in (0.0, -1.0, float("nan"), 1e9):
        with pytest.raises(Exception):
            ctx.set_wait_limit(bad)
