"""The lean front layout against the all-resident one.

With every front resident, a parent reads its children's contribution
blocks in place and the solves read the panels from the fronts.  The lean
layout reuses a front's memory once its parent has assembled its
contribution block (placement by lifetime) and keeps the factored panels in a
compact panel pool -- the device-side counterpart of the reference's
contribution-block arena (src/multifrontal.jl:180-187, 321-332).  The
arithmetic is the same, so factors and solutions must be bitwise identical,
and the working memory must shrink.
"""

import numpy as np
import pytest

from pureumfpack import PRECISION_FP64, PRECISION_MIXED, GpuContext, colamd_order, row_scaling, symbolic_mf
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


def _run(A, S, Rs, precision, lean):
    ctx = GpuContext(precision=precision, lean_fronts=lean)
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, Rs, True) == 0
    B = M.rhs(A.n, seed=6, nrhs=5)
    X = ctx.solve(B, 1)
    L, U, p, q, pinv = ctx.factors()
    return ctx.stats(), L, U, p, X


CASES = [
    ("poisson3d-20", lambda: M.poisson3d(20), False),
    ("convdiff-16-colamd", lambda: M.convdiff3d(16), True),
    ("random-3000-colamd", lambda: M.random_unsym(3000, 5, 10.0, seed=3), True),
]


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name,make,colamd", CASES, ids=[c[0] for c in CASES])
def test_lean_layout_is_bitwise_identical(name, make, colamd, precision):
    A = make()
    S = symbolic_mf(A, q=colamd_order(A) if colamd else None)
    Rs = row_scaling(A, 2 if colamd else 1)
    st0, L0, U0, p0, X0 = _run(A, S, Rs, precision, False)
    st1, L1, U1, p1, X1 = _run(A, S, Rs, precision, True)
    assert st0["lean"] is False and st1["lean"] is True
    np.testing.assert_array_equal(p1, p0)
    np.testing.assert_array_equal(L1.rowval, L0.rowval)
    np.testing.assert_array_equal(L1.nzval, L0.nzval)
    np.testing.assert_array_equal(U1.nzval, U0.nzval)
    np.testing.assert_array_equal(X1, X0)
    assert st1["pool_elems"] < st0["pool_elems"] + st0["front_elems_full"]


def test_lean_layout_shrinks_working_memory_of_a_deep_tree():
    A = M.random_unsym(3000, 5, 10.0, seed=3)
    S = symbolic_mf(A, q=colamd_order(A))
    ctx = GpuContext(lean_fronts=True, merge_fronts=False)
    ctx.analyze(A, S)
    st = ctx.stats()
    # the resident layout needs the sum of nf^2; the lean pool (working fronts
    # + panels + inverses) needs a fraction of it (one front per supernode:
    # merged fronts make this tree shallow)
    assert st["pool_elems"] < 0.5 * st["front_elems_full"], (st["pool_elems"], st["front_elems_full"])
