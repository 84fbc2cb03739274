"""Merged fronts (the default) on the GPU: chains of supernodes factored as
one front must give the reference's factorization exactly as the one-front-
per-supernode path does -- the same fill, L/U patterns and pivot sequence
(src/multifrontal.jl:247-263 searches pivots only among a supernode's own
pivot rows, and the merged front keeps that restriction per original
supernode), values to the parity tolerance, and solutions to the oracle's.
The matrices include strongly pivoting ones (small diagonal shift), whose
merged pivot blocks span several supernodes, and pivot blocks larger than
the shared-memory panel (the global-memory pivot search)."""

import numpy as np
import pytest

from helpers import assert_close_values, assert_same_structure, column_value_errors, reconstruction_error
from oracle import oracle as O
from pureumfpack import PRECISION_MIXED, GpuContext, colamd_order, symbolic_mf
from pureumfpack import matrices as M
from pureumfpack.api import GPLUFactorization

pytestmark = pytest.mark.gpu


def factor(A, q, merge, precision=0, lean=False):
    ctx = GpuContext(merge_fronts=merge, precision=precision, lean_fronts=lean)
    ctx.analyze(A, symbolic_mf(A, q=q))
    assert ctx.factor(A.nzval, None, False) == 0
    return GPLUFactorization(ctx)


CASES = [
    ("poisson3d-14", lambda: M.poisson3d(14), False, True),
    ("convdiff-12-colamd", lambda: M.convdiff3d(12), True, True),
    ("poisson2d-60", lambda: M.poisson2d(60), False, True),
    ("pivoting-2500-amd", lambda: M.random_unsym(2500, 5, 1.0, seed=7), False, False),
    ("pivoting-2500-colamd", lambda: M.random_unsym(2500, 5, 1.0, seed=7), True, False),
]


@pytest.mark.parametrize("name,make,use_colamd,well_conditioned", CASES, ids=[c[0] for c in CASES])
def test_merged_fronts_match_oracle(name, make, use_colamd, well_conditioned):
    A = make()
    q = colamd_order(A) if use_colamd else None
    fo = O.multifrontal_lu(A, q=q, check=False)
    Fm = factor(A, q, True)
    Fu = factor(A, q, False)
    sm, su = Fm.ctx.stats(), Fu.ctx.stats()
    assert sm["merged"] and sm["fronts"] < sm["nsuper"] == su["nsuper"] == su["fronts"]
    for F in (Fm, Fu):
        assert_same_structure(fo, F.L, F.U, F.p, F.q, F.pinv)
        # the reference tests' bound (test/multifrontal_test.jl:38-39) for the
        # well-conditioned matrices; element growth scales it for the others
        assert reconstruction_error(A, F.L, F.U, F.p, F.q) <= (1e-9 if well_conditioned else 1e-7)
    if well_conditioned:
        assert_close_values(fo, Fm.L, Fm.U)
    else:
        # element growth amplifies the rounding differences of the operation
        # orders (about 1e-10 normwise for these matrices, over a thousand
        # off-diagonal pivots each)
        for F in (Fm, Fu):
            assert_close_values(fo, F.L, F.U, rtol=1e-8, entry_rtol=1e-5)
    nl, _ = column_value_errors(Fu.L.colptr, Fu.L.nzval, Fm.L.nzval)
    nu, _ = column_value_errors(Fu.U.colptr, Fu.U.nzval, Fm.U.nzval)
    assert max(nl, nu) <= (1e-12 if well_conditioned else 1e-8), f"merged vs single fronts {max(nl, nu):.2e}"


def test_merged_fronts_lean_layout_and_solve():
    A = M.convdiff3d(14)
    q = colamd_order(A)
    fo = O.multifrontal_lu(A, q=q, check=False)
    F = factor(A, q, True, lean=True)
    assert F.ctx.stats()["lean"]
    assert_same_structure(fo, F.L, F.U, F.p, F.q, F.pinv)
    assert_close_values(fo, F.L, F.U)
    B = M.rhs(A.n, seed=3, nrhs=2)
    x = F.ctx.solve(B, 1)
    S = A.to_scipy()
    assert np.linalg.norm(S @ x - B) <= 1e-12 * np.linalg.norm(B) * 1e3


def test_merged_fronts_mixed_precision_refines_to_fp64():
    A = M.poisson3d(16)
    F = factor(A, None, True, precision=PRECISION_MIXED)
    assert F.ctx.stats()["merged"]
    B = M.rhs(A.n, seed=5, nrhs=3)
    x = F.ctx.solve(B, 3)
    S = A.to_scipy()
    r = B - S @ x
    eta = np.max(np.abs(r).max(0) / (np.abs(S).sum(1).max() * np.abs(x).max(0) + np.abs(B).max(0)))
    assert eta <= 1e-14
