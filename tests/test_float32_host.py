"""Float32 matrices (the reference's generic Tv = Float32), host side.

The oracle's Float32 path -- row scaling, sgetrf / strsm / sgemm fronts and
the solve with refinement, all in Float32 -- meets the reference's own
Float32 check (bench/mf_verify.jl:33-37: residual <= 1e-3 for
sprand(Float32, 400, 400, 10/400) + 5I) and keeps the Float64 path's
structure; libmfgpu's host row scaling of a Float32 matrix is bitwise the
oracle's (Float32 sums in storage order, scaling.jl:92-115 with
R = Float32)."""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O
from pureumfpack import SCALE_MAX, SCALE_NONE, SCALE_SUM, SparseCSC, row_scaling
from pureumfpack import matrices as M


def sprand32(n, density, shift, seed):
    S = sp.random(n, n, density=density, random_state=seed, dtype=np.float32) + shift * sp.eye(n, dtype=np.float32)
    return SparseCSC.from_scipy(S.astype(np.float32))


@pytest.mark.parametrize("kind", [SCALE_NONE, SCALE_SUM, SCALE_MAX])
def test_row_scaling_f32_is_the_oracles(kind):
    A = M.convdiff3d(6).astype(np.float32)
    rs = row_scaling(A, kind)
    assert rs.dtype == np.float32
    np.testing.assert_array_equal(rs, O.row_scaling_f32(A, int(kind)))


@pytest.mark.parametrize("name,make", [("sprand-400", lambda: sprand32(400, 10 / 400, 5.0, 1)),
                                       ("poisson3d-8", lambda: M.poisson3d(8).astype(np.float32))])
def test_oracle_float32_path(name, make):
    A = make()
    assert A.nzval.dtype == np.float32
    F = O.splu_f32(A)
    Fd = O.splu(A.astype(np.float64))
    np.testing.assert_array_equal(F.F.Lcolptr, Fd.F.Lcolptr)
    np.testing.assert_array_equal(F.F.Ucolptr, Fd.F.Ucolptr)
    # Float32 values differ from the Float64 factorization at Float32 rounding
    err = np.linalg.norm(F.F.Lnzval - Fd.F.Lnzval) / np.linalg.norm(Fd.F.Lnzval)
    assert err <= 1e-5
    b = np.random.default_rng(3).standard_normal(A.n).astype(np.float32)
    x = O.solve_f32(F, b)
    assert x.dtype == np.float32
    S = A.to_scipy()
    assert np.linalg.norm(S @ x - b) / np.linalg.norm(b) <= 1e-3
