"""Batched systems on the GPU against the oracle, system by system.

A batch goes through one handle: every system keeps its own ordering,
symbolic structure, pivots and factors, so each one must match the oracle's
splu(A_i; method=:multifrontal) (src/interface.jl:93-120) exactly in
structure and to the factor-value rule of tests/helpers.py, and its
solutions must match solve(F_i, b_i; refine) (src/interface.jl:170-177).
"""

import numpy as np
import pytest

from helpers import assert_close_values, assert_same_structure
from oracle import oracle as O
from pureumfpack import (
    PRECISION_MIXED,
    SCALE_MAX,
    SCALE_SUM,
    SingularException,
    SparseCSC,
    colamd_order,
    splu_batch,
)
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


def _small_batch(count=24, seed=5):
    # the batch generator's mix at reduced sides: 2-D U[4, 24], 3-D U[3, 9]
    rng = np.random.default_rng(seed)
    out = []
    for t in range(count):
        A = M.poisson2d(int(rng.integers(4, 25))) if t % 2 == 0 else M.poisson3d(int(rng.integers(3, 10)))
        A = A.add_diagonal(float(rng.random()))
        out.append((A, rng.standard_normal((A.n, 4))))
    return out


def _eta(A, x, b):
    r = b - A.to_scipy() @ x
    anorm = np.max(np.abs(A.to_scipy()).sum(axis=1))
    return float(np.max(np.abs(r).max(axis=0) / (anorm * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))))


def test_batch_factors_match_oracle_per_system():
    sysl = _small_batch()
    As = [A for A, _ in sysl]
    F = splu_batch(As, scale=SCALE_SUM)
    assert len(F) == len(As) and not np.any(F.status)
    for i, A in enumerate(As):
        Fo = O.splu(A, scale=int(SCALE_SUM))
        L, U, p, q, pinv = F.factors(i)
        np.testing.assert_array_equal(F.Rs[i], Fo.Rs)
        assert_same_structure(Fo.F, L, U, p, q, pinv)
        assert_close_values(Fo.F, L, U)


def test_batch_solve_matches_oracle_per_system():
    sysl = _small_batch(count=16, seed=9)
    As = [A for A, _ in sysl]
    Bs = [B for _, B in sysl]
    F = splu_batch(As)
    Xs = F.solve(Bs, refine=2)
    for A, B, X in zip(As, Bs, Xs):
        Xo = O.solve(O.splu(A), B, refine=2)
        assert np.linalg.norm(X - Xo) <= 1e-10 * np.linalg.norm(Xo)
        assert _eta(A, X, B) <= 1e-14
    # a single right-hand side per system
    x1 = F.solve([B[:, 0] for B in Bs])
    for A, B, x in zip(As, Bs, x1):
        assert x.shape == (A.n,)
        assert _eta(A, x[:, None], B[:, :1]) <= 1e-13


def test_batch_colamd_scale_max_matches_oracle():
    As = [M.convdiff3d(5), M.random_unsym(300, 5, 10.0, seed=1), M.convdiff3d(6), M.random_unsym(150, 5, 10.0, seed=2)]
    F = splu_batch(As, scale=SCALE_MAX, ordering="colamd")
    for i, A in enumerate(As):
        Rs = O.row_scaling(A, int(SCALE_MAX))
        fo = O.multifrontal_lu(O.apply_row_scaling(A, Rs), q=colamd_order(A), check=False)
        L, U, p, q, pinv = F.factors(i)
        assert_same_structure(fo, L, U, p, q, pinv)
        assert_close_values(fo, L, U, entry_rtol=1e-10)


def test_batch_reports_singular_systems():
    ok = M.poisson2d(5)
    # [[1, 1], [1, 1]]: zero pivot at factor column 2
    sing = SparseCSC.from_coo([1, 2, 1, 2], [1, 1, 2, 2], [1.0, 1.0, 1.0, 1.0], 2, 2)
    As = [ok, sing, ok, sing]
    with pytest.raises(SingularException) as e:
        splu_batch(As, scale=0)
    assert e.value.info == 2
    F = splu_batch(As, scale=0, check=False)
    np.testing.assert_array_equal(F.status, [0, 2, 0, 2])


def test_batch_mixed_precision_reaches_fp64_accuracy():
    sysl = _small_batch(count=12, seed=11)
    As = [A for A, _ in sysl]
    Bs = [B for _, B in sysl]
    F = splu_batch(As, precision=PRECISION_MIXED)
    Xs = F.solve(Bs, refine=3)
    for A, B, X in zip(As, Bs, Xs):
        assert _eta(A, X, B) <= 1e-14
