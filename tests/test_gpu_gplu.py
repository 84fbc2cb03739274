"""Gilbert-Peierls LU on the GPU against the oracle's restatement of
src/gplu.jl:173-303 (tests/test_gplu_oracle.py pins the oracle).

The device factorization does the reference's arithmetic in the reference's
order (depth-first reach order, first-position pivot ties, every product and
difference rounded on its own), so the factors, the pivots and the solutions
must equal the oracle's bit for bit: Lcolptr / Lrowval / Lnzval, the same for
U, p, q and pinv, and x from solve(F, b; refine).  Cases follow the
reference's GP-LU tests (test/pureumfpack_test.jl:11-123,
test/multifrontal_test.jl:12-21, test/robustness.jl:38-42,
test/interfaces.jl): the orderings and scalings of splu(A; method=:gplu),
tol 0 / 0.1 / 1 (threshold and strict partial pivoting), sort_factors off,
singular matrices, a batch of independent systems, factors that outgrow
their first segment, and the reference's generic element types
(test/robustness.jl:8-26): ComplexF64 in Julia's complex arithmetic and
Float32 end to end.
"""

import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from pureumfpack import (SCALE_MAX, SCALE_NONE, SCALE_SUM, ArgumentError, BatchGPLU, DimensionMismatch, GpluContext,
                         SingularException, SparseCSC, gplu, solve, splu, symbolic_mf)
from pureumfpack import matrices as M

pytestmark = pytest.mark.gpu


def sprand_plus(n, density, shift, seed):
    """sparse(sprand(n, n, density) + shift * I) with numpy's generator."""
    rng = np.random.default_rng(seed)
    idx = rng.choice(n * n, size=int(round(density * n * n)), replace=False)
    I, J = idx % n + 1, idx // n + 1
    d = np.arange(1, n + 1)
    return SparseCSC.from_coo(np.concatenate([I, d]), np.concatenate([J, d]),
                              np.concatenate([rng.random(len(idx)), np.full(n, float(shift))]), n, n)


def assert_bitwise(Fo, L, U, p, q, pinv):
    np.testing.assert_array_equal(L.colptr, Fo.Lcolptr)
    np.testing.assert_array_equal(L.rowval, Fo.Lrowval)
    np.testing.assert_array_equal(L.nzval, Fo.Lnzval)
    np.testing.assert_array_equal(U.colptr, Fo.Ucolptr)
    np.testing.assert_array_equal(U.rowval, Fo.Urowval)
    np.testing.assert_array_equal(U.nzval, Fo.Unzval)
    np.testing.assert_array_equal(p, Fo.p)
    np.testing.assert_array_equal(q, Fo.q)
    np.testing.assert_array_equal(pinv, Fo.pinv)


CASES = [
    ("poisson2d-16", lambda: M.poisson2d(16), "amd", 0.1, SCALE_SUM),
    ("poisson3d-8", lambda: M.poisson3d(8), "amd", 0.1, SCALE_SUM),
    ("randmat-300", lambda: M.randmat(300, 6), "colamd", 0.1, SCALE_MAX),
    ("arrowband-300", lambda: M.arrowband(300, 4), "natural", 1.0, SCALE_NONE),
    ("convdiff-8", lambda: M.convdiff3d(8), "colamd", 0.1, SCALE_SUM),
    ("grid3d-random-7", lambda: M.grid3d_random(7), "amd", 1.0, SCALE_NONE),
    ("sprand-200", lambda: sprand_plus(200, 10 / 200, 1.0, 5), "natural", 1.0, SCALE_NONE),
    ("random-unsym-800", lambda: M.random_unsym(800, 5, 10.0, 3), "colamd", 0.1, SCALE_MAX),
]


@pytest.mark.parametrize("name,make,ordering,tol,scale", CASES, ids=[c[0] for c in CASES])
def test_splu_gplu_matches_oracle_bitwise(name, make, ordering, tol, scale):
    A = make()
    Fo = O.splu_gplu(A, ordering=ordering, tol=tol, scale=scale)
    F = splu(A, method="gplu", ordering=ordering, tol=tol, scale=scale)
    np.testing.assert_array_equal(F.Rs, Fo.Rs)
    assert_bitwise(Fo.F, *F.ctx.factors())
    B = M.rhs(A.n, 11, 3)
    for refine in (0, 2):
        np.testing.assert_array_equal(solve(F, B, refine=refine), O.solve(Fo, B, refine=refine))


@pytest.mark.parametrize("tol", [0.0, 0.1, 1.0])
@pytest.mark.parametrize("sort_factors", [True, False])
def test_gplu_tol_and_sorting(tol, sort_factors):
    A = sprand_plus(120, 10 / 120, 1.0, seed=int(tol * 10) + 3)
    q = O.colamd_order(A)
    Fo = O.gplu(A, q=q, tol=tol, sort_factors=sort_factors)
    F = gplu(A, q=q, tol=tol, sort_factors=sort_factors)
    assert_bitwise(Fo, F.L, F.U, F.p, F.q, F.pinv)
    b = M.rhs(A.n, 5)
    np.testing.assert_array_equal(F.ldiv(b), O.solve_raw(Fo, b))


def test_gplu_published_fill():
    """predicted_fill(S) == nnz(gplu(M; q = S.qf, tol = 0)) at the published
    poisson2d-32 fill (results/SUMMARY.md:32, test/multifrontal_test.jl:43-51)."""
    A = M.poisson2d(32)
    S = symbolic_mf(A)
    F = gplu(A, q=S.qf, tol=0.0)
    assert len(F.L.rowval) + len(F.U.rowval) == 23800
    assert_bitwise(O.gplu(A, q=S.qf, tol=0.0), F.L, F.U, F.p, F.q, F.pinv)


def test_gplu_doctests():
    """src/gplu.jl:36-41, :159-166; test/interfaces.jl."""
    A = SparseCSC.from_coo([1, 2, 1, 2], [1, 1, 2, 2], [2.0, 1.0, 1.0, 2.0], 2, 2)
    F = gplu(A)
    Ad = A.to_scipy().toarray()
    assert np.array_equal(F.L.to_scipy().toarray() @ F.U.to_scipy().toarray(), Ad[F.p - 1][:, F.q - 1])
    np.testing.assert_array_equal(gplu(A, tol=1.0).ldiv(np.array([1.0, 0.0])),
                                  [0.6666666666666666, -0.3333333333333333])
    assert F.size() == (2, 2)
    np.testing.assert_allclose(splu(A).ldiv(np.array([1.0, 0.0])), np.linalg.solve(Ad, [1.0, 0.0]), rtol=1e-15)


def test_gplu_edge_cases():
    """test/pureumfpack_test.jl:114-122 (splu's default method is :gplu)."""
    A1 = SparseCSC.from_coo([1], [1], [3.0], 1, 1)
    assert splu(A1).ldiv(np.array([6.0]))[0] == 2.0
    D = SparseCSC.from_coo([1, 2, 3, 4], [1, 2, 3, 4], [2.0, 3.0, 5.0, 7.0], 4, 4)
    np.testing.assert_array_equal(splu(D).ldiv(np.array([2.0, 6.0, 15.0, 28.0])), [1.0, 2.0, 3.0, 4.0])
    with pytest.raises(DimensionMismatch):
        gplu(SparseCSC.from_coo([1, 2], [1, 1], [1.0, 1.0], 2, 1))
    with pytest.raises(ArgumentError):
        splu(D, method="gplu", ordering="nonsense")


def test_gplu_singular():
    """test/robustness.jl:38-42, and check = false on the same matrices."""
    A = SparseCSC.from_coo([1, 2, 1, 2], [1, 1, 2, 2], [1.0, 2.0, 2.0, 4.0], 2, 2)
    with pytest.raises(SingularException) as e:
        gplu(A, tol=1.0, check=True)
    assert e.value.info == 2
    B = SparseCSC.from_coo([1, 3], [1, 3], [1.0, 1.0], 3, 3)
    with pytest.raises(SingularException) as e:
        splu(B, method="gplu", ordering="natural", scale=SCALE_NONE)
    assert e.value.info == 2
    # check = false goes on with a zero pivot, as the reference does
    F = gplu(A, tol=1.0, check=False)
    assert_bitwise(O.gplu(A, tol=1.0, check=False), F.L, F.U, F.p, F.q, F.pinv)
    # ... unless the pivot rows stop being a permutation (invperm throws)
    C = SparseCSC.from_coo([2, 2], [1, 2], [1.0, 1.0], 2, 2)
    with pytest.raises(RuntimeError):
        O.gplu(C, check=False)
    with pytest.raises(ArgumentError):
        gplu(C, check=False)


def small_batch(count, seed):
    """Shifted grid Laplacians as the batched workload draws them, at smaller
    sides: 2-D sides U[4, 24], 3-D sides U[3, 9], shift U[0, 1]."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(count):
        A = M.poisson2d(int(rng.integers(4, 25))) if t % 2 == 0 else M.poisson3d(int(rng.integers(3, 10)))
        out.append(A.add_diagonal(float(rng.random())))
    return out


@pytest.mark.parametrize("initial_capacity", [0, 16])
def test_batch_matches_oracle_bitwise(initial_capacity):
    """Every system of a batch as splu(A_i; method=:gplu) alone; with a
    16-entry first segment every system but the smallest outgrows it and is
    factored again."""
    As = small_batch(40, 7)
    As.insert(5, SparseCSC(0, 0, np.ones(1, np.int64), np.zeros(0, np.int64), np.zeros(0)))
    Fb = BatchGPLU(As, ordering="amd", tol=0.1, scale=SCALE_SUM, initial_capacity=initial_capacity)
    assert not Fb.status.any()
    t = Fb.ctx.timings()
    if initial_capacity:
        assert t["reruns"] > 0 and t["factor_launches"] > 1
    Bs = [M.rhs(A.n, i, 4) if A.n else np.zeros((0, 4)) for i, A in enumerate(As)]
    Xs = Fb.solve(Bs, refine=1)
    for i, A in enumerate(As):
        if A.n == 0:
            continue
        Fo = O.splu_gplu(A, ordering="amd", tol=0.1, scale=SCALE_SUM)
        assert_bitwise(Fo.F, *Fb.factors(i))
        np.testing.assert_array_equal(Xs[i], O.solve(Fo, Bs[i], refine=1))


def test_context_reuse_and_state():
    """A handle refactors in place; solving before a factorization is an error."""
    ctx = GpluContext()
    with pytest.raises(Exception):
        ctx.solve(np.ones(3))
    A = M.poisson2d(10)
    for tol in (0.1, 1.0):
        st = ctx.factor([A], [O.amd_order_sym(A)], None, tol=tol)
        assert st[0] == 0
        assert_bitwise(O.gplu(A, q=O.amd_order_sym(A), tol=tol), *ctx.factors())
    with pytest.raises(ArgumentError):
        bad = SparseCSC(2, 2, np.array([1, 3, 4]), np.array([2, 1, 2]), np.ones(3))   # rows not ascending
        ctx.factor([bad])


# -- the reference's generic Tv: ComplexF64 and Float32 (test/robustness.jl) --
def sprand_c(n, density, shift, seed):
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    nnz = rng.binomial(n * n, density)
    I, J = rng.integers(0, n, nnz), rng.integers(0, n, nnz)
    V = rng.random(nnz) + 1j * rng.random(nnz)
    return (sp.coo_matrix((V, (I, J)), shape=(n, n)).tocsc() + shift * sp.eye(n, format="csc")).tocsc()


def grid_c(k, seed):
    """Complex values on the 3-D grid pattern with a weak diagonal: row
    interchanges under tol = 1."""
    import scipy.sparse as sp

    S = M.poisson3d(k).to_scipy().tocoo()
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(S.nnz) + 1j * rng.standard_normal(S.nnz)
    return sp.csc_matrix((v, (S.row, S.col)), shape=S.shape)


def crandn(n, seed, k=None):
    rng = np.random.default_rng(seed)
    shape = (n,) if k is None else (n, k)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("ordering", ["amd", "colamd", "natural"])
def test_complex_splu_matches_oracle_bitwise(ordering):
    """test/robustness.jl:8-17 (splu's default method on ComplexF64)."""
    S = sprand_c(400, 8 / 400, 5.0, 7)
    A, Ao = SparseCSC.from_scipy(S), O.ComplexCSC.from_scipy(S)
    Fo = O.splu_gplu(Ao, ordering=ordering)
    F = splu(A, ordering=ordering)
    np.testing.assert_array_equal(F.Rs, Fo.Rs)
    assert_bitwise(Fo.F, *F.ctx.factors())
    b = crandn(400, 8)
    for refine in (0, 1):
        x = solve(F, b, refine=refine)
        np.testing.assert_array_equal(x, O.solve_gplu(Fo, b, refine=refine))
        assert np.linalg.norm(S @ x - b) / np.linalg.norm(b) <= 1e-10


@pytest.mark.parametrize("tol", [0.1, 1.0])
def test_complex_grid_with_interchanges(tol):
    S = grid_c(7, 3)
    A, Ao = SparseCSC.from_scipy(S), O.ComplexCSC.from_scipy(S)
    q = O.amd_order_sym(Ao)
    Fo = O.gplu(Ao, q=q, tol=tol)
    F = gplu(A, q=q, tol=tol)
    assert not np.array_equal(Fo.p, Fo.q)   # rows were interchanged
    assert_bitwise(Fo, F.L, F.U, F.p, F.q, F.pinv)
    B = crandn(A.n, 4, 3)
    np.testing.assert_array_equal(F.ldiv(B), O.solve_gplu(Fo, B))


def test_float32_splu_matches_oracle_bitwise():
    """test/robustness.jl:18-26: a Float32 matrix is factored and solved in
    Float32 (x is Float32, residual <= 1e-4)."""
    n = 300
    rng = np.random.default_rng(9)
    nnz = rng.binomial(n * n, 8 / n)
    I, J = rng.integers(1, n + 1, nnz), rng.integers(1, n + 1, nnz)
    d = np.arange(1, n + 1)
    A = SparseCSC.from_coo(np.concatenate([I, d]), np.concatenate([J, d]),
                           np.concatenate([rng.random(nnz), np.full(n, 5.0)]), n, n).astype(np.float32)
    b = rng.standard_normal(n).astype(np.float32)
    Fo = O.splu_gplu(A, ordering="amd")
    F = splu(A, ordering="amd")
    assert F.Rs.dtype == np.float32
    L, U, p, q, pinv = F.ctx.factors()
    assert L.nzval.dtype == np.float32
    assert_bitwise(Fo.F, SparseCSC(n, n, L.colptr, L.rowval, L.nzval.astype(np.float64)),
                   SparseCSC(n, n, U.colptr, U.rowval, U.nzval.astype(np.float64)), p, q, pinv)
    for refine in (0, 2):
        x = solve(F, b, refine=refine)
        assert x.dtype == np.float32
        np.testing.assert_array_equal(x, O.solve_gplu(Fo, b, refine=refine))
    x = F.ldiv(b)
    assert np.linalg.norm(A.to_scipy().astype(np.float64) @ x - b) / np.linalg.norm(b) <= 1e-4


def test_complex_batch_and_type_checks():
    """A batch of complex systems, each as splu(A_i) alone; the handle's
    real-valued calls refuse its complex factors."""
    Ss = [sprand_c(60 + 13 * i, 6 / (60 + 13 * i), 4.0, 20 + i) for i in range(6)] + [grid_c(5, 9)]
    As = [SparseCSC.from_scipy(S) for S in Ss]
    Fb = BatchGPLU(As, ordering="colamd", tol=0.1, scale=SCALE_MAX)
    Bs = [crandn(A.n, 30 + i, 2) for i, A in enumerate(As)]
    Xs = Fb.solve(Bs, refine=1)
    for i, S in enumerate(Ss):
        Fo = O.splu_gplu(O.ComplexCSC.from_scipy(S), ordering="colamd", tol=0.1, scale=O.SCALE_MAX)
        assert_bitwise(Fo.F, *Fb.factors(i))
        np.testing.assert_array_equal(Xs[i], O.solve_gplu(Fo, Bs[i], refine=1))
    ctx = Fb.ctx
    n = As[0].n
    out = np.empty(n + 1, np.int64)
    rc = ctx._lib.mfgpu_gplu_get_factors(ctx._h, 0, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), None, None,
                                         None, None, None, None, None, None)
    assert rc == -4   # MFGPU_ERR_STATE: complex factors, real fetch
    with pytest.raises(ArgumentError):   # one element type per batch
        ctx.factor([As[0], SparseCSC.from_scipy(Ss[1].real)])
