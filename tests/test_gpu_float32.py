"""Float32 matrices on the GPU (the reference's generic Tv = Float32).

splu / multifrontal_lu of a Float32 matrix factor it with Float32 fronts and
return Float32 factors: the row scaling is bitwise the oracle's Float32 one,
fill, L/U patterns and the pivot sequence are the oracle's Float32
factorization's, and values agree to Float32 rounding (the large updates
run as BF16x3 tensor-core products, the oracle's as sgemm).  Solves meet the
reference's Float32 check (bench/mf_verify.jl:33-37, residual <= 1e-3) and
agree with the oracle's Float32 solve."""

import numpy as np
import pytest
import scipy.sparse as sp

from helpers import assert_same_structure, column_value_errors
from oracle import oracle as O
from pureumfpack import SparseCSC, multifrontal_lu, solve, splu
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


def sprand32(n, density, shift, seed):
    S = sp.random(n, n, density=density, random_state=seed, dtype=np.float32) + shift * sp.eye(n, dtype=np.float32)
    return SparseCSC.from_scipy(S.astype(np.float32))


CASES = [
    ("sprand-400", lambda: sprand32(400, 10 / 400, 5.0, 1)),
    ("poisson3d-12", lambda: M.poisson3d(12).astype(np.float32)),
    ("convdiff-12", lambda: M.convdiff3d(12).astype(np.float32)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_float32_splu_matches_oracle(name, make):
    A = make()
    fo = O.splu_f32(A)
    F = splu(A, method="multifrontal")
    np.testing.assert_array_equal(F.Rs, fo.Rs)
    L, U = F.L, F.U
    assert L.nzval.dtype == np.float32 and U.nzval.dtype == np.float32
    assert_same_structure(fo.F, L, U, F.p, F.q, F._f._get()[4])
    nl, _ = column_value_errors(fo.F.Lcolptr, fo.F.Lnzval, L.nzval.astype(np.float64))
    nu, _ = column_value_errors(fo.F.Ucolptr, fo.F.Unzval, U.nzval.astype(np.float64))
    assert max(nl, nu) <= 1e-4, (nl, nu)
    b = np.random.default_rng(7).standard_normal(A.n).astype(np.float32)
    S = A.to_scipy()
    x = solve(F, b)
    assert x.dtype == np.float32
    assert np.linalg.norm(S @ x - b) / np.linalg.norm(b) <= 1e-3
    xo = O.solve_f32(fo, b)
    assert np.linalg.norm(x - xo) <= 1e-4 * np.linalg.norm(xo)
    x2 = solve(F, b, refine=2)
    assert np.linalg.norm(S.astype(np.float64) @ x2.astype(np.float64) - b) <= 1e-5 * np.linalg.norm(b)


def test_float32_multifrontal_lu_ldiv():
    A = M.poisson2d(30).astype(np.float32)
    F = multifrontal_lu(A)
    assert F.L.nzval.dtype == np.float32
    b = np.random.default_rng(2).standard_normal(A.n).astype(np.float32)
    x = F.ldiv(b)
    assert x.dtype == np.float32
    assert np.linalg.norm(A.to_scipy() @ x - b) / np.linalg.norm(b) <= 1e-3
