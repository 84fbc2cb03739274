"""GPU parity at the benchmark configurations' full sizes.

The smaller parity suites stop at a few thousand unknowns; these run the
factorizations the benchmark configurations time, where the large-front code
runs (1,024-pivot merged fronts, pivot blocks of thousands of rows, the
speculative panels and their pivoting rerun, long-K tensor-core tiles):

* poisson3d(48) + 1e-3 I, AMD, SCALE_SUM: splu(A; method=:multifrontal)
  against the oracle's (src/interface.jl:93-120): fill, patterns, p, q, pinv
  bit-identical, values within 1e-12 (tests/helpers.py rule); the mixed
  form's FP32 factors with the identical structure and FP32-level values;
* convdiff3d(40), SCALE_MAX, with COLAMD through multifrontal_lu(As;
  q=colamd_order(A)) (src/multifrontal.jl:152) and with the reference-exact
  splu route (AMD; splu ignores `ordering`, src/interface.jl:103-105);
* random 20,000 x 20,000 + 10 I, COLAMD, SCALE_MAX: its reference structure
  needs 309 G front elements, beyond the oracle, so the GPU factors are
  checked against the pattern the symbolic analysis fixes
  (helpers.symbolic_pattern, itself pinned to the oracle on the CPU) and by
  backward error;
* 64 seeded systems of the 1,024-system batch against the oracle, each.
"""

import numpy as np
import pytest

from helpers import assert_close_values, assert_same_structure, assert_structure_from_symbolic, backward_error
from oracle import oracle as O
from pureumfpack import (
    PRECISION_MIXED,
    SCALE_MAX,
    SCALE_SUM,
    colamd_order,
    solve,
    splu,
    splu_batch,
    splu_q,
    symbolic_mf,
)
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu

# FP32 fronts (BF16x3 tensor-core products with FP32 accumulation) against
# the FP64 oracle: per-column normwise agreement at FP32 level times the
# element growth and accumulation length of these fronts.
MIXED_COLWISE = 1e-4


def _c2():
    return M.poisson3d(48).add_diagonal(1e-3)


def test_c2_poisson3d_48_shift_fp64_matches_oracle():
    A = _c2()
    Fo = O.splu(A, scale=int(SCALE_SUM), check=False)
    F = splu(A, method="multifrontal", scale=SCALE_SUM)
    np.testing.assert_array_equal(F.Rs, Fo.Rs)
    assert_same_structure(Fo.F, F.L, F.U, F.p, F.q, F._f._get()[4])
    assert int(F.L.colptr[-1] - 1 + F.U.colptr[-1] - 1) == int(Fo.F.Lcolptr[-1] - 1 + Fo.F.Ucolptr[-1] - 1)
    assert_close_values(Fo.F, F.L, F.U)
    b = M.rhs(A.n, seed=1)
    x = solve(F, b, refine=1)
    assert backward_error(A, x, b) <= 1e-14


def test_c2_poisson3d_48_shift_mixed_structure_and_values():
    A = _c2()
    Fo = O.splu(A, scale=int(SCALE_SUM), check=False)
    F = splu(A, method="multifrontal", scale=SCALE_SUM, precision=PRECISION_MIXED)
    assert not F.ctx.stats()["refactored_fp64"]
    assert_same_structure(Fo.F, F.L, F.U, F.p, F.q, F._f._get()[4])
    assert_close_values(Fo.F, F.L, F.U, rtol=MIXED_COLWISE, entry_rtol=1.0)
    b = M.rhs(A.n, seed=1)
    x = solve(F, b, refine=2)
    assert backward_error(A, x, b) <= 1e-14


def test_c4a_convdiff_40_colamd_matches_oracle():
    A = M.convdiff3d(40)
    q = colamd_order(A)
    Rs = O.row_scaling(A, int(SCALE_MAX))
    fo = O.multifrontal_lu(O.apply_row_scaling(A, Rs), q=q, check=False)
    F = splu_q(A, q, scale=SCALE_MAX)
    np.testing.assert_array_equal(F.Rs, Rs)
    assert_same_structure(fo, F.L, F.U, F.p, F.q, F._f._get()[4])
    assert_close_values(fo, F.L, F.U, entry_rtol=1e-10)
    b = M.rhs(A.n, seed=2)
    x = solve(F, b, refine=1)
    assert backward_error(A, x, b) <= 1e-14


def test_c4a_convdiff_40_splu_reference_route_matches_oracle():
    A = M.convdiff3d(40)
    Fo = O.splu(A, scale=int(SCALE_MAX), check=False)
    F = splu(A, method="multifrontal", ordering="colamd", tol=0.1, scale=SCALE_MAX)
    np.testing.assert_array_equal(F.Rs, Fo.Rs)
    assert_same_structure(Fo.F, F.L, F.U, F.p, F.q, F._f._get()[4])
    assert_close_values(Fo.F, F.L, F.U, entry_rtol=1e-10)


def test_c4b_random_20000_structure_from_symbolic():
    A = M.random_unsym(20000, 5, 10.0, seed=3)
    q = colamd_order(A)
    S = symbolic_mf(A, q=q)
    F = splu_q(A, q, scale=SCALE_MAX)
    assert_structure_from_symbolic(S, F.L, F.U, F.p)
    np.testing.assert_array_equal(F.q, S.qf)
    np.testing.assert_array_equal(F.Rs, O.row_scaling(A, int(SCALE_MAX)))
    b = M.rhs(A.n, seed=3)
    x = solve(F, b, refine=1)
    assert backward_error(A, x, b) <= 1e-14


def test_c3_batch_sample_matches_oracle():
    sysl = M.batched_set(1024, seed=0, nrhs=4)
    As = [A for A, _ in sysl]
    F = splu_batch(As, scale=SCALE_SUM)
    assert not np.any(F.status)
    pick = np.sort(np.random.default_rng(64).choice(len(As), size=64, replace=False))
    for i in pick:
        A = As[i]
        Fo = O.splu(A, scale=int(SCALE_SUM), check=False)
        L, U, p, q, pinv = F.factors(int(i))
        np.testing.assert_array_equal(F.Rs[i], Fo.Rs)
        assert_same_structure(Fo.F, L, U, p, q, pinv)
        assert_close_values(Fo.F, L, U)
    Xs = F.solve([B for _, B in sysl], refine=1)
    for i in pick:
        A, B = sysl[i]
        assert backward_error(A, Xs[i], B) <= 1e-14
