"""libmfgpu's host ordering and symbolic analysis: identical to the oracle (CPU)."""

import numpy as np
import pytest

from oracle import oracle as O
from pureumfpack import amd_order_sym, colamd_order, predicted_fill, row_scaling, symbolic_mf
from pureumfpack import matrices as M

MATS = [
    ("poisson2d-16", lambda: M.poisson2d(16)),
    ("poisson2d-100", lambda: M.poisson2d(100)),
    ("poisson3d-8", lambda: M.poisson3d(8)),
    ("poisson3d-20", lambda: M.poisson3d(20)),
    ("randmat-400", lambda: M.randmat(400, 6)),
    ("arrowband-400", lambda: M.arrowband(400, 4)),
    ("convdiff-12", lambda: M.convdiff3d(12)),
    ("random-3000", lambda: M.random_unsym(3000, 5, 10.0, seed=1)),
    ("n1", lambda: M.poisson2d(1)),
    ("n4", lambda: M.poisson2d(2)),
]


@pytest.mark.parametrize("name,make", MATS, ids=[m[0] for m in MATS])
def test_orderings_identical(name, make):
    A = make()
    np.testing.assert_array_equal(amd_order_sym(A), O.amd_order_sym(A))
    np.testing.assert_array_equal(colamd_order(A), O.colamd_order(A))


@pytest.mark.parametrize("name,make", MATS, ids=[m[0] for m in MATS])
@pytest.mark.parametrize("use_colamd", [False, True])
def test_symbolic_identical(name, make, use_colamd):
    A = make()
    q = O.colamd_order(A) if use_colamd else None
    So = O.symbolic_mf(A, q=q)
    S = symbolic_mf(A, q=q)
    np.testing.assert_array_equal(S.qf, So.qf)
    np.testing.assert_array_equal(S.parent, So.parent)
    np.testing.assert_array_equal(S.sstart, So.sstart)
    np.testing.assert_array_equal(S.colcount, np.diff(So.cs_ptr))
    np.testing.assert_array_equal(S.child_ptr, So.ch_ptr)
    np.testing.assert_array_equal(S.child_idx, So.ch_idx)
    assert predicted_fill(S) == O.predicted_fill(So)
    for j in range(1, A.n + 1, max(1, A.n // 97)):
        np.testing.assert_array_equal(S.colstruct(j), So.colstruct(j))


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_row_scaling_identical(kind):
    A = M.random_unsym(2000, 5, 1.0, seed=2)
    np.testing.assert_array_equal(row_scaling(A, kind), O.row_scaling(A, kind))


def test_fill_kat_64():
    """Product symbolic on the 64^3 workload (too slow for the oracle's
    column-by-column structure pass in a CPU test): supernode partition and
    fill are self-consistent and the order is a permutation."""
    A = M.poisson3d(24)
    S = symbolic_mf(A)
    assert predicted_fill(S) == 3749118
    assert S.nsuper == 9348
    assert np.array_equal(np.sort(S.qf), np.arange(1, A.n + 1))


def test_short_order_is_rejected_before_the_library():
    """A caller's q reaches the C ABI as a bare pointer: a short one is a
    DimensionMismatch on the host, never a read past its end."""
    from pureumfpack import DimensionMismatch, SparseCSC, symbolic_mf

    A = SparseCSC.from_coo([1, 2, 3], [1, 2, 3], [1.0, 2.0, 3.0], 3, 3)
    with pytest.raises(DimensionMismatch):
        symbolic_mf(A, q=[1, 2])
