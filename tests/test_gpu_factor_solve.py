"""mfgpu_factor_solve: factor + solve(b; refine) in one call.

The right-hand sides are copied to the device on their own stream while the
factorization runs; the solution must be that of mfgpu_factor followed by
mfgpu_solve, bit for bit, for the FP64 and the mixed form, with page-locked
and with ordinary host buffers, and a singular matrix must return its
singular column (SingularException's argument) without solving.
"""

import numpy as np
import pytest

from pureumfpack import PRECISION_FP64, PRECISION_MIXED, GpuContext, SparseCSC, row_scaling, symbolic_mf
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,refine", [(PRECISION_FP64, 0), (PRECISION_FP64, 1), (PRECISION_MIXED, 2)],
                         ids=["fp64", "fp64-refine", "mixed"])
@pytest.mark.parametrize("pinned", [False, True], ids=["pageable", "pinned"])
def test_factor_solve_is_factor_then_solve(precision, refine, pinned):
    import torch

    A = M.poisson3d(16)
    S = symbolic_mf(A)
    Rs = row_scaling(A, 1)
    B = M.rhs(A.n, seed=21, nrhs=9)
    ref = GpuContext(device=0, precision=precision)
    ref.analyze(A, S)
    assert ref.factor(A.nzval, Rs, True) == 0
    x_ref = ref.solve(B, refine)
    ctx = GpuContext(device=0, precision=precision)
    ctx.analyze(A, S)
    if pinned:
        Bp = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).pin_memory().numpy().reshape(B.shape, order="F")
    else:
        Bp = B
    for _ in range(2):   # twice: the same buffers and graphs again
        st, x = ctx.factor_solve(A.nzval, Rs, Bp, refine)
        assert st == 0
        np.testing.assert_array_equal(x, x_ref)


def test_factor_solve_reports_a_singular_column():
    # [[1, 1], [1, 1]]: zero pivot at factor column 2
    A = SparseCSC.from_coo([1, 2, 1, 2], [1, 1, 2, 2], [1.0, 1.0, 1.0, 1.0], 2, 2)
    ctx = GpuContext(device=0)
    ctx.analyze(A, symbolic_mf(A))
    st, x = ctx.factor_solve(A.nzval, None, np.ones(2), 0, check=True)
    assert st == 2 and x is None
