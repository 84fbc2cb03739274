"""ComplexF64 matrices on the GPU against the oracle's ComplexF64 restatement.

The reference's generic Tv covers ComplexF64 (test/multifrontal_test.jl:63-75,
test/robustness.jl:8-18, bench/mf_verify.jl:27-31): Julia's lu! / rdiv! /
ldiv! / mul! on complex front blocks, i.e. LAPACK zgetrf (pivot: the first
largest |re| + |im|) / ztrsm / zgemm.  libmfgpu factors complex fronts on the
GPU (mfgpu_factor_c64): fill, patterns, p, q and pinv must equal the oracle's
(tests/test_complex_host.py pins the oracle), values agree per column to
1e-12, and solve(F, b; refine) agrees with the oracle's and reaches the
reference tests' residual bounds.  Matrices are seeded stand-ins with the
reference tests' shapes: sprand(ComplexF64, n, n, 8/n) + 5I, its Hermitian
pattern Ac + Ac', and complex values on the 3-D grid pattern (large fronts
and pivot blocks, row interchanges inside them).
"""

import numpy as np
import pytest
import scipy.sparse as sp

from helpers import assert_close_values, assert_same_structure
from oracle import oracle as O
from pureumfpack import GpuContext, MfgpuError, SparseCSC, colamd_order, row_scaling, solve, splu, symbolic_mf
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


def sprand_c(n, density, seed, shift=5.0):
    rng = np.random.default_rng(seed)
    nnz = rng.binomial(n * n, density)
    I = rng.integers(0, n, nnz)
    J = rng.integers(0, n, nnz)
    V = rng.random(nnz) + 1j * rng.random(nnz)
    return (sp.coo_matrix((V, (I, J)), shape=(n, n)).tocsc() + shift * sp.eye(n, format="csc")).tocsc()


def grid_c(k, seed):
    """The 3-D 7-point pattern with complex values: diagonal in U[1, 2] +
    U[0, 1] i, off-diagonals N(0, 0.25) + N(0, 0.25) i -- row interchanges
    inside the pivot blocks of large fronts."""
    S = M.poisson3d(k).to_scipy().tocoo()
    rng = np.random.default_rng(seed)
    v = 0.5 * (rng.standard_normal(S.nnz) + 1j * rng.standard_normal(S.nnz))
    d = S.row == S.col
    v[d] = rng.uniform(1, 2, d.sum()) + 1j * rng.random(d.sum())
    return sp.csc_matrix((v, (S.row, S.col)), shape=S.shape)


def crandn(n, seed, k=None):
    rng = np.random.default_rng(seed)
    shape = (n,) if k is None else (n, k)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


CASES = [
    ("hermitian-pattern-300", lambda: (lambda S: (S + S.conj().T).tocsc())(sprand_c(300, 8 / 300, 11)), None),
    ("sprand-1200", lambda: sprand_c(1200, 8 / 1200, 7), None),
    ("sprand-1200-colamd", lambda: sprand_c(1200, 8 / 1200, 7), "colamd"),
    ("grid-10", lambda: grid_c(10, 3), None),
    ("grid-14", lambda: grid_c(14, 5), None),
]


def _gpu_factor(A, q, scale, merge):
    S = symbolic_mf(A, q=q)
    Rs = row_scaling(A, scale)
    ctx = GpuContext(device=0, merge_fronts=merge)
    ctx.analyze(A, S)
    ctx.factor_c64(A.nzval, Rs if scale else None, False)
    return ctx, Rs


@pytest.mark.parametrize("merge", [True, False], ids=["merged", "unmerged"])
@pytest.mark.parametrize("name,make,order", CASES, ids=[c[0] for c in CASES])
def test_complex_factors_match_oracle(name, make, order, merge):
    Ssp = make()
    A = SparseCSC.from_scipy(Ssp)
    Ao = O.ComplexCSC.from_scipy(Ssp)
    q = colamd_order(A) if order == "colamd" else None
    for scale in (O.SCALE_SUM, O.SCALE_NONE):
        Fo = O.splu_c64(Ao, scale=scale, q=q, check=False)
        ctx, Rs = _gpu_factor(A, q, scale, merge)
        np.testing.assert_array_equal(Rs, Fo.Rs)
        L, U, p, qq, pinv = ctx.factors()
        assert L.nzval.dtype == np.complex128
        assert_same_structure(Fo.F, L, U, p, qq, pinv)
        assert_close_values(Fo.F, L, U, entry_rtol=1e-10)
    if name.startswith("grid"):
        assert np.sum(p != qq) > 5, "case meant to exercise row interchanges"


@pytest.mark.parametrize("name,make,order", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_complex_solve_matches_oracle(name, make, order):
    Ssp = make()
    A = SparseCSC.from_scipy(Ssp)
    Ao = O.ComplexCSC.from_scipy(Ssp)
    b = crandn(A.n, 12)
    B = crandn(A.n, 13, k=5)
    F = splu(A, method="multifrontal")
    Fo = O.splu_c64(Ao)
    for rhs in (b, B):
        for refine in (0, 1):
            x = solve(F, rhs, refine=refine)
            xo = O.solve_c64(Fo, rhs, refine=refine)
            assert x.dtype == np.complex128 and x.shape == rhs.shape
            assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)
            r = Ssp @ x - rhs
            assert np.linalg.norm(r) <= 1e-12 * np.linalg.norm(rhs)   # the reference tests ask 1e-8 / 1e-10
    x = F.ldiv(b)   # F \ b
    assert np.linalg.norm(Ssp @ x - b) <= 1e-12 * np.linalg.norm(b)


def test_real_and_complex_entry_points_do_not_mix():
    from pureumfpack import _lib as L

    Ssp = sprand_c(200, 8 / 200, 3)
    A = SparseCSC.from_scipy(Ssp)
    F = splu(A, method="multifrontal")
    ctx = F.ctx
    n = A.n
    x = np.zeros(n)
    with pytest.raises(MfgpuError) as e:   # real solve on complex factors
        ctx._check(ctx._lib.mfgpu_solve(ctx._h, 1, L.ptr(x, L.f64p), n, L.ptr(x, L.f64p), n, 0))
    assert e.value.code == -4
    # a real matrix on the same handle is factored as real again
    Ar = SparseCSC(n, n, A.colptr, A.rowval, A.nzval.real.copy())
    ctx.factor(Ar.nzval, row_scaling(Ar, 1), False)
    assert not np.iscomplexobj(ctx.factors()[0].nzval)
    with pytest.raises(MfgpuError) as e:   # complex solve on real factors
        ctx._check(ctx._lib.mfgpu_solve_c64(ctx._h, 1, L.ptr(x, L.f64p), L.ptr(x, L.f64p), 0))
    assert e.value.code == -4
