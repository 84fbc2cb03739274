"""GPU solves against the oracle (src/interface.jl:123-177, src/solve.jl:10-79).

The GPU solve walks the same factors supernode by supernode; the oracle
sweeps them CSC column by column.  Both are backward stable, so solutions
agree to cond(A) * eps; the tests require the reference's own residual bounds
(test/multifrontal_test.jl:53-61) plus agreement with the oracle's solution.
"""

import numpy as np
import pytest

from helpers import backward_error
from oracle import oracle as O
from pureumfpack import PRECISION_FP64, PRECISION_MIXED, SCALE_MAX, SCALE_NONE, SCALE_SUM, multifrontal_lu, solve, splu
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu

SOLVE_CASES = [
    ("poisson2d-30", lambda: M.poisson2d(30)),
    ("poisson2d-100", lambda: M.poisson2d(100)),
    ("poisson3d-8", lambda: M.poisson3d(8)),
    ("poisson3d-12", lambda: M.poisson3d(12)),
    ("poisson3d-20", lambda: M.poisson3d(20)),
    ("randmat-800", lambda: M.randmat(800, 6)),
    ("convdiff-12", lambda: M.convdiff3d(12)),
]


@pytest.mark.parametrize("name,make", SOLVE_CASES, ids=[c[0] for c in SOLVE_CASES])
def test_splu_solve_matches_oracle(name, make):
    A = make()
    b = M.rhs(A.n, seed=0)
    F = splu(A, method="multifrontal")
    Fo = O.splu(A)
    for refine in (0, 2):
        x = solve(F, b, refine=refine)
        xo = O.solve(Fo, b, refine=refine)
        assert np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b) <= 1e-8
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-10
    assert backward_error(A, x, b) <= 1e-14


def test_raw_factorization_solve():
    A = M.poisson3d(10)
    b = M.rhs(A.n, seed=1)
    F = multifrontal_lu(A)
    x = F.ldiv(b)
    xo = O.solve_raw(O.multifrontal_lu(A), b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-12


@pytest.mark.parametrize("scale", [SCALE_NONE, SCALE_SUM, SCALE_MAX])
def test_scalings(scale):
    # test/multifrontal_test.jl:63-69
    A = M.poisson3d(8)
    b = M.rhs(A.n, seed=2)
    x = solve(splu(A, method="multifrontal", scale=scale), b)
    assert np.linalg.norm(A.matvec(x) - b) / np.linalg.norm(b) <= 1e-8


@pytest.mark.parametrize("nrhs", [4, 37, 256])
def test_multiple_rhs_equal_per_column(nrhs):
    A = M.poisson3d(12)
    B = M.rhs(A.n, seed=4, nrhs=nrhs)
    F = splu(A, method="multifrontal")
    X = solve(F, B, refine=1)
    for c in (0, nrhs // 2, nrhs - 1):
        xc = solve(F, np.ascontiguousarray(B[:, c]), refine=1)
        assert np.linalg.norm(X[:, c] - xc) <= 1e-13 * np.linalg.norm(xc)
    assert backward_error(A, X, B) <= 1e-14


@pytest.mark.parametrize("precision,refine", [(PRECISION_FP64, 0), (PRECISION_MIXED, 2)], ids=["fp64", "mixed"])
def test_many_rhs_large_fronts_match_oracle(precision, refine):
    # Many right-hand sides on fronts with hundreds of pivots: the solve runs
    # its row-parallel pull assembly and gather, K-chunked top-level products
    # with their fold, the thin-supernode and leaf kernels and the few-row
    # product tiles, and the mixed form's factorization the bulk-copy GEMM;
    # the solutions must agree with the oracle's solve(F, B; refine)
    # (src/interface.jl:170-177) and reach the accuracy target.
    from pureumfpack import GpuContext, row_scaling, symbolic_mf

    A = M.poisson3d(28)
    B = M.rhs(A.n, seed=9, nrhs=96)
    S = symbolic_mf(A)
    Rs = row_scaling(A, 1)
    ctx = GpuContext(device=0, precision=precision)
    ctx.analyze(A, S)
    assert ctx.factor(A.nzval, Rs, True) == 0
    X = ctx.solve(B, refine)
    Xo = O.solve(O.splu(A), B, refine=max(refine, 1))
    assert np.linalg.norm(X - Xo) <= 1e-10 * np.linalg.norm(Xo)
    assert backward_error(A, X, B) <= 1e-14
    np.testing.assert_array_equal(ctx.solve(B, refine), X)   # deterministic: the same bits again


def test_refinement_does_not_degrade():
    # test/pureumfpack_test.jl:105-112 through the multifrontal path
    A = M.random_unsym(1500, 5, 1.0, seed=5)
    b = M.rhs(A.n, seed=6)
    F = splu(A, method="multifrontal")
    r0 = np.linalg.norm(A.matvec(solve(F, b)) - b)
    r2 = np.linalg.norm(A.matvec(solve(F, b, refine=2)) - b)
    assert r2 <= r0 + 1e-12
