"""The oracle's Gilbert-Peierls LU (src/gplu.jl:173-303) against the
reference's own tests and golden values (CPU).

Pins: the doctests of src/gplu.jl (2 x 2 reconstruction and solve), the
published fill counts (results/SUMMARY.md:32-36 in tests/golden/kat.json)
through the reference's fill identity predicted_fill(S) ==
nnz(gplu(M; q = S.qf, tol = 0)) (test/multifrontal_test.jl:12-21, 43-51), the
reconstruction, strict-pivoting, sort_factors, canonical-CSC and
singularity tests of test/pureumfpack_test.jl:11-57 and
test/robustness.jl:38-42, splu(A; method = :gplu) end to end over the
orderings and scalings (test/pureumfpack_test.jl:80-123), and the generic
element types of test/robustness.jl:8-26 (ComplexF64 through every
ordering, Float32 staying Float32).
"""

import json
import os

import numpy as np
import pytest

from helpers import reconstruction_error
from oracle import oracle as O
from pureumfpack import SparseCSC
from pureumfpack import matrices as M

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kat.json")))


def _factors(A, F):
    L = SparseCSC(A.n, A.n, F.Lcolptr, F.Lrowval, F.Lnzval)
    U = SparseCSC(A.n, A.n, F.Ucolptr, F.Urowval, F.Unzval)
    return L, U


def sprand_plus(n, density, shift, seed):
    """sparse(sprand(n, n, density) + shift * I) with numpy's generator."""
    rng = np.random.default_rng(seed)
    nnz = int(round(density * n * n))
    idx = rng.choice(n * n, size=min(nnz, n * n), replace=False)
    I, J = idx % n + 1, idx // n + 1
    V = rng.random(len(idx))
    d = np.arange(1, n + 1)
    return SparseCSC.from_coo(np.concatenate([I, d]), np.concatenate([J, d]),
                              np.concatenate([V, np.full(n, float(shift))]), n, n)


def test_gplu_doctests():
    """src/gplu.jl:36-41 and :159-166, src/solve.jl:55-60."""
    A = SparseCSC.from_coo([1, 2, 1, 2], [1, 1, 2, 2], [2.0, 1.0, 1.0, 2.0], 2, 2)
    F = O.gplu(A)
    L, U = _factors(A, F)
    Ap = A.to_scipy().toarray()[F.p - 1][:, F.q - 1]
    assert np.array_equal(L.to_scipy().toarray() @ U.to_scipy().toarray(), Ap)
    x = O.solve_raw(O.gplu(A, tol=1.0), np.array([1.0, 0.0]))
    np.testing.assert_array_equal(x, GOLDEN["solve_2x2"])


@pytest.mark.parametrize("case", [c for c in GOLDEN["fill"] if c["fill"] < 2_000_000],
                         ids=[c["matrix"] for c in GOLDEN["fill"] if c["fill"] < 2_000_000])
def test_gplu_fill_is_the_published_fill(case):
    kind, k = case["matrix"].split("-")
    A = (M.poisson2d if kind == "poisson2d" else M.poisson3d)(int(k))
    S = O.symbolic_mf(A)
    F = O.gplu(A, q=S.qf, tol=0.0)
    assert len(F.Lrowval) + len(F.Urowval) == case["fill"]


@pytest.mark.parametrize("make", [lambda: M.poisson2d(16), lambda: M.poisson3d(8), lambda: M.randmat(400, 6)])
def test_gplu_fill_equals_multifrontal_fill(make):
    A = make()
    Msym = A + A.transpose()
    S = O.symbolic_mf(Msym)
    Fg = O.gplu(Msym, q=S.qf, tol=0.0)
    Fm = O.multifrontal_lu(Msym, check=False)
    assert len(Fg.Lrowval) + len(Fg.Urowval) == O.predicted_fill(S)
    assert len(Fg.Lrowval) + len(Fg.Urowval) == len(Fm.Lrowval) + len(Fm.Urowval)


@pytest.mark.parametrize("n", [1, 2, 10, 64, 300])
@pytest.mark.parametrize("trial", [0, 1])
def test_gplu_reconstruction(n, trial):
    A = sprand_plus(n, min(1.0, 8 / n), n, seed=100 * n + trial)
    F = O.gplu(A, tol=0.1)
    L, U = _factors(A, F)
    Ld = L.to_scipy().toarray()
    Ud = U.to_scipy().toarray()
    assert np.array_equal(np.tril(Ld), Ld) and np.all(np.diag(Ld) == 1.0)
    assert np.array_equal(np.triu(Ud), Ud)
    assert np.array_equal(np.sort(F.p), np.arange(1, n + 1))
    assert np.array_equal(np.sort(F.q), np.arange(1, n + 1))
    assert reconstruction_error(A, L, U, F.p, F.q) <= 1e-9


@pytest.mark.parametrize("n", [50, 200])
def test_gplu_strict_partial_pivoting(n):
    A = sprand_plus(n, 10 / n, 1.0, seed=n)
    F = O.gplu(A, tol=1.0)
    assert np.max(np.abs(F.Lnzval)) <= 1.0
    b = np.random.default_rng(n).standard_normal(n)
    x = O.solve_raw(F, b)
    r = A.to_scipy() @ x - b
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-8


def test_gplu_unsorted_factors_still_solve():
    A = sprand_plus(120, 10 / 120, 5.0, seed=7)
    b = np.random.default_rng(7).standard_normal(120)
    Fs = O.gplu(A, tol=0.1, sort_factors=True)
    Fu = O.gplu(A, tol=0.1, sort_factors=False)
    xs, xu = O.solve_raw(Fs, b), O.solve_raw(Fu, b)
    assert np.linalg.norm(xs - xu) <= 1e-10 * np.linalg.norm(xs)
    # same entries, only the order inside each column differs
    for cp, a, b_ in ((Fs.Lcolptr, Fs.Lrowval, Fu.Lrowval), (Fs.Ucolptr, Fs.Urowval, Fu.Urowval)):
        assert np.array_equal(Fs.Lcolptr, Fu.Lcolptr) and np.array_equal(Fs.Ucolptr, Fu.Ucolptr)
        for j in range(120):
            s = slice(cp[j] - 1, cp[j + 1] - 1)
            assert np.array_equal(a[s], np.sort(b_[s]))


@pytest.mark.parametrize("make", [lambda: M.poisson3d(8), lambda: M.randmat(400, 10), lambda: M.arrowband(400, 4)])
def test_gplu_sorted_factors_are_canonical(make):
    A = make()
    F = O.gplu(A, q=O.amd_order_sym(A), tol=0.1)
    for cp, ri in ((F.Lcolptr, F.Lrowval), (F.Ucolptr, F.Urowval)):
        for j in range(A.n):
            assert np.all(np.diff(ri[cp[j] - 1:cp[j + 1] - 1]) > 0)


def test_gplu_singular():
    """test/robustness.jl:38-42."""
    A = SparseCSC.from_coo([1, 2, 1, 2], [1, 1, 2, 2], [1.0, 2.0, 2.0, 4.0], 2, 2)
    with pytest.raises(O.SingularException) as e:
        O.gplu(A, tol=1.0, check=True)
    assert e.value.info == 2
    B = SparseCSC.from_coo([1, 3], [1, 3], [1.0, 1.0], 3, 3)
    with pytest.raises(O.SingularException):
        O.splu_gplu(B, ordering="natural", scale=O.SCALE_NONE)


@pytest.mark.parametrize("make", [lambda: M.poisson2d(30), lambda: M.poisson3d(10), lambda: M.randmat(800, 8),
                                  lambda: M.arrowband(800, 4)])
def test_splu_gplu_orderings_and_scalings(make):
    A = make()
    b = np.random.default_rng(A.n).standard_normal(A.n)
    xref = np.linalg.solve(A.to_scipy().toarray(), b)
    for ordering in ("natural", "amd", "colamd"):
        for scale in (O.SCALE_NONE, O.SCALE_SUM, O.SCALE_MAX):
            F = O.splu_gplu(A, ordering=ordering, tol=0.1, scale=scale)
            x = O.solve(F, b)
            assert np.linalg.norm(A.to_scipy() @ x - b) / np.linalg.norm(b) <= 1e-8
            assert np.linalg.norm(x - xref) / np.linalg.norm(xref) <= 1e-6


def sprand_complex(n, density, shift, seed):
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    nnz = rng.binomial(n * n, density)
    I, J = rng.integers(0, n, nnz), rng.integers(0, n, nnz)
    V = rng.random(nnz) + 1j * rng.random(nnz)
    return (sp.coo_matrix((V, (I, J)), shape=(n, n)).tocsc() + shift * sp.eye(n, format="csc")).tocsc()


@pytest.mark.parametrize("ordering", ["amd", "colamd", "natural"])
def test_gplu_complex_robustness(ordering):
    """test/robustness.jl:8-17: splu(A::SparseMatrixCSC{ComplexF64}; ordering) \\ b
    (the default method, :gplu) to residual 1e-10, and against a direct solve."""
    import scipy.sparse.linalg as spla

    S = sprand_complex(400, 8 / 400, 5.0, 7)
    A = O.ComplexCSC.from_scipy(S)
    rng = np.random.default_rng(8)
    b = rng.standard_normal(400) + 1j * rng.standard_normal(400)
    F = O.splu_gplu(A, ordering=ordering)
    x = O.solve_gplu(F, b)
    assert np.linalg.norm(S @ x - b) / np.linalg.norm(b) <= 1e-10
    xr = spla.spsolve(S, b)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-9
    L = F.F
    for cp, ri in ((L.Lcolptr, L.Lrowval), (L.Ucolptr, L.Urowval)):
        assert all(np.all(np.diff(ri[cp[j] - 1:cp[j + 1] - 1]) > 0) for j in range(400))
    # the raw factor solves A[p, q] x = b too
    Fr = O.gplu(A, q=O.gplu_order(A, ordering))
    xr2 = O.solve_gplu(Fr, b)
    assert np.linalg.norm(S @ xr2 - b) / np.linalg.norm(b) <= 1e-10


def test_gplu_float32_robustness():
    """test/robustness.jl:18-26: a Float32 matrix stays Float32 end to end."""
    n = 300
    rng = np.random.default_rng(9)
    nnz = rng.binomial(n * n, 8 / n)
    I, J = rng.integers(1, n + 1, nnz), rng.integers(1, n + 1, nnz)
    d = np.arange(1, n + 1)
    A = SparseCSC.from_coo(np.concatenate([I, d]), np.concatenate([J, d]),
                           np.concatenate([rng.random(nnz), np.full(n, 5.0)]), n, n)
    A = SparseCSC(n, n, A.colptr, A.rowval, A.nzval.astype(np.float32))
    b = rng.standard_normal(n).astype(np.float32)
    F = O.splu_gplu(A, ordering="amd")
    x = O.solve_gplu(F, b)
    assert x.dtype == np.float32
    assert np.linalg.norm(A.to_scipy().astype(np.float64) @ x - b) / np.linalg.norm(b) <= 1e-4
    # the Float32 values are Float32 numbers (widened exactly) and differ from the Float64 factorization's
    F64 = O.splu_gplu(SparseCSC(n, n, A.colptr, A.rowval, A.nzval.astype(np.float64)), ordering="amd")
    assert np.array_equal(F.F.Lnzval.astype(np.float32).astype(np.float64), F.F.Lnzval)
    assert not np.array_equal(F.F.Lnzval, F64.F.Lnzval)
