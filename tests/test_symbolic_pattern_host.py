"""The factor pattern that the symbolic analysis fixes, pinned to the oracle.

helpers.symbolic_pattern derives, from symbolic_mf alone, L's and U's column
pointers, U's rows, the relabelled pivot-block rows of L and the update rows
of L before relabelling (src/multifrontal.jl:73-104, 278-317, 347-357).  The
GPU test of the 20,000-unknown random matrix (whose reference structure is
beyond the oracle's reach) checks its factors against it; here it is checked
against the oracle's own factorizations, with and without row interchanges.
"""

import numpy as np
import pytest

from helpers import assert_structure_from_symbolic, symbolic_pattern
from oracle import oracle as O
from pureumfpack import SparseCSC, colamd_order, symbolic_mf
from pureumfpack import matrices as M

CASES = [
    ("convdiff-6-amd", lambda: M.convdiff3d(6), False),
    ("poisson3d-10-amd", lambda: M.poisson3d(10), False),
    ("random-2000-colamd", lambda: M.random_unsym(2000, 5, 10.0, seed=3), True),
    ("random-1500-pivoting", lambda: M.random_unsym(1500, 5, 1.0, seed=4), True),
    ("random-3000-pivoting", lambda: M.random_unsym(3000, 4, 0.5, seed=7), True),
    ("grid3d-random-10", lambda: M.grid3d_random(10, 0.5, seed=1), False),
]


@pytest.mark.parametrize("name,make,colamd", CASES, ids=[c[0] for c in CASES])
def test_symbolic_pattern_is_the_oracles(name, make, colamd):
    A = make()
    q = colamd_order(A) if colamd else None
    S = symbolic_mf(A, q=q)
    fo = O.multifrontal_lu(A, q=q, check=False)
    L = SparseCSC(A.n, A.n, fo.Lcolptr, fo.Lrowval, fo.Lnzval)
    U = SparseCSC(A.n, A.n, fo.Ucolptr, fo.Urowval, fo.Unzval)
    assert_structure_from_symbolic(S, L, U, fo.p)
    if "pivoting" in name:
        assert np.sum(fo.p != S.qf) > 100, "case meant to exercise row interchanges"


def test_symbolic_pattern_detects_a_wrong_pivot_block():
    A = M.random_unsym(1500, 5, 1.0, seed=4)
    q = colamd_order(A)
    S = symbolic_mf(A, q=q)
    fo = O.multifrontal_lu(A, q=q, check=False)
    L = SparseCSC(A.n, A.n, fo.Lcolptr, fo.Lrowval, fo.Lnzval)
    U = SparseCSC(A.n, A.n, fo.Ucolptr, fo.Urowval, fo.Unzval)
    # a row permutation that crosses two supernodes' pivot blocks
    ss = np.asarray(S.sstart) - 1
    a, b = int(ss[3]), int(ss[-2])
    p = fo.p.copy()
    p[[a, b]] = p[[b, a]]
    with pytest.raises(AssertionError):
        assert_structure_from_symbolic(S, L, U, p)
    E = symbolic_pattern(S)
    assert E["Urowval"].size == fo.Urowval.size
