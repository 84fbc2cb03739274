"""ComplexF64 through the multifrontal path: the oracle's restatement, pinned.

The reference's generic Tv covers ComplexF64 (test/multifrontal_test.jl:63-75,
test/robustness.jl:8-18, bench/mf_verify.jl:27-31): its fronts go through
Julia's lu! / rdiv! / ldiv! / mul! on a Matrix{ComplexF64}, i.e. LAPACK
zgetrf / ztrsm / zgemm, and the oracle makes the same calls.  Pinned here
against the reference tests' own bounds, a sparse direct solver (scipy's
SuperLU), the factorization identity (Rs .* A)[p, q] == L * U, the pattern
of the Float64 path, and LAPACK's complex pivot rule (largest |re| + |im|,
which differs from the largest modulus).  Matrices are seeded stand-ins with
the reference tests' shapes and value distribution: sprand(ComplexF64, n, n,
8/n) draws uniform [0, 1) real and imaginary parts, plus 5I.

The last test runs the device algorithm on complex values through
tests/plan_emulator.cpp (the library's own plan: merged fronts with the
pivot search kept inside each original supernode, assembly and extend-add
maps, CSC scatter) and checks it against the oracle's ComplexF64
factorization: the plan and the pivot rule carry over to complex fronts.
"""

import ctypes

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from helpers import column_value_errors
from oracle import oracle as O
from pureumfpack.sparse import SparseCSC


def sprand_c(n, density, seed, shift=5.0):
    rng = np.random.default_rng(seed)
    nnz = rng.binomial(n * n, density)
    I = rng.integers(0, n, nnz)
    J = rng.integers(0, n, nnz)
    V = rng.random(nnz) + 1j * rng.random(nnz)
    return (sp.coo_matrix((V, (I, J)), shape=(n, n)).tocsc() + shift * sp.eye(n, format="csc")).tocsc()


def crandn(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def rel_resid(S, x, b):
    return np.linalg.norm(S @ x - b) / np.linalg.norm(b)


@pytest.mark.parametrize("scale", [O.SCALE_NONE, O.SCALE_SUM, O.SCALE_MAX])
def test_hermitian_pattern_matrix(scale):
    # test/multifrontal_test.jl:70-74: Ac + Ac', residual <= 1e-8
    S = sprand_c(300, 8 / 300, seed=11)
    S = (S + S.conj().T).tocsc()
    A = O.ComplexCSC.from_scipy(S)
    b = crandn(300, seed=12)
    x = O.solve_c64(O.splu_c64(A, scale=scale), b)
    assert rel_resid(S, x, b) <= 1e-8
    assert rel_resid(S, x, b) <= 1e-13   # what the oracle actually reaches


@pytest.mark.parametrize("ordering", ["amd", "colamd", "natural"])
def test_orderings_against_a_sparse_direct_solver(ordering):
    # test/robustness.jl:8-18: residual <= 1e-10, and within 1e-9 of lu(A) \ b
    n = 400
    S = sprand_c(n, 8 / n, seed=7)
    A = O.ComplexCSC.from_scipy(S)
    q = {"amd": None, "colamd": O.colamd_order(A), "natural": np.arange(1, n + 1)}[ordering]
    b = crandn(n, seed=8)
    x = O.solve_c64(O.splu_c64(A, q=q), b)
    assert rel_resid(S, x, b) <= 1e-10
    xr = sla.spsolve(S, b)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) <= 1e-9


def _csc(colptr, rowval, nzval, n):
    return sp.csc_matrix((nzval, rowval - 1, colptr - 1), shape=(n, n))


@pytest.mark.parametrize("scale", [O.SCALE_NONE, O.SCALE_SUM])
def test_factorization_identity(scale):
    # (Rs .* A)[p, q] == L * U (src/interface.jl:38-48)
    n = 500
    S = sprand_c(n, 6 / n, seed=21)
    A = O.ComplexCSC.from_scipy(S)
    P = O.splu_c64(A, scale=scale)
    F = P.F
    L = _csc(F.Lcolptr, F.Lrowval, F.Lnzval, n)
    U = _csc(F.Ucolptr, F.Urowval, F.Unzval, n)
    SA = sp.diags(P.Rs) @ S
    lhs = SA.tocsr()[F.p - 1, :].tocsc()[:, F.q - 1]
    err = abs(lhs - L @ U).max() / abs(SA).max()
    assert err <= 1e-14
    # L unit lower with the diagonal stored first, U upper with it stored last
    assert np.all(F.Lnzval[F.Lcolptr[:-1] - 1] == 1.0)
    assert np.all(F.Urowval[F.Ucolptr[1:] - 2] == np.arange(1, n + 1))


def test_pattern_is_the_float64_paths():
    # the symbolic structure depends only on the pattern: the column pointers,
    # U's rows and the column order equal the Float64 factorization's
    n = 400
    S = sprand_c(n, 8 / n, seed=31)
    A = O.ComplexCSC.from_scipy(S)
    Fc = O.multifrontal_lu_c64(A)
    Ar = SparseCSC(n, n, A.colptr, A.rowval, np.abs(A.nzval))
    Fr = O.multifrontal_lu(Ar)
    for key in ("Lcolptr", "Ucolptr", "Urowval", "q"):
        np.testing.assert_array_equal(getattr(Fc, key), getattr(Fr, key), err_msg=key)


@pytest.mark.parametrize("a,b,first", [
    # |1+1i| = 1.414 < 1.45 but |re| + |im| = 2 > 1.45: LAPACK keeps row 1
    (1 + 1j, 1.45 + 0j, 1),
    # mirrored: LAPACK takes row 2, a largest-modulus rule would keep row 1
    (1.45 + 0j, 1 + 1j, 2),
])
def test_pivot_rule_is_lapacks(a, b, first):
    S = sp.csc_matrix(np.array([[a, 0.25], [b, 1.0]], dtype=np.complex128))
    A = O.ComplexCSC.from_scipy(S)
    F = O.multifrontal_lu_c64(A, q=np.array([1, 2]), check=True)
    assert F.p[0] == first


@pytest.mark.parametrize("kind", [O.SCALE_SUM, O.SCALE_MAX])
def test_row_scaling_uses_the_modulus(kind):
    # scaling.jl:92-115 with R = Float64: abs(z) = hypot(re, im), in CSC order
    S = sprand_c(300, 8 / 300, seed=41)
    A = O.ComplexCSC.from_scipy(S)
    Rs = O.row_scaling_c64(A, kind)
    acc = np.zeros(A.n)
    mag = np.hypot(A.nzval.real, A.nzval.imag)
    if kind == O.SCALE_SUM:
        np.add.at(acc, A.rowval - 1, mag)
    else:
        np.maximum.at(acc, A.rowval - 1, mag)
    np.testing.assert_array_equal(Rs, np.where(acc > 0, 1.0 / np.where(acc > 0, acc, 1.0), 1.0))


def test_singular_column_matches_the_float64_path():
    # a stored zero pivot (the structure of test/multifrontal_test.jl's
    # singular case): SingularException at the same column as Float64's
    n = 6
    colptr = np.array([1, 2, 4, 5, 6, 7, 8])
    rowval = np.array([1, 1, 2, 3, 4, 5, 6])
    vals = np.array([2, 1 + 1j, 3, 0, 7, 1, 4], dtype=np.complex128) * (1 + 0.5j)
    A = O.ComplexCSC(n, n, colptr, rowval, vals)
    assert A.nzval[3] == 0
    with pytest.raises(O.SingularException) as ec:
        O.multifrontal_lu_c64(A, check=True)
    Ar = SparseCSC(n, n, colptr, rowval, np.abs(vals))
    with pytest.raises(O.SingularException) as er:
        O.multifrontal_lu(Ar, check=True)
    assert ec.value.info == er.value.info


def test_refinement_and_many_right_hand_sides():
    n = 400
    S = sprand_c(n, 8 / n, seed=51)
    A = O.ComplexCSC.from_scipy(S)
    F = O.splu_c64(A)
    B = np.stack([crandn(n, seed=60 + k) for k in range(3)], axis=1)
    X0 = O.solve_c64(F, B)
    X2 = O.solve_c64(F, B, refine=2)
    for k in range(3):
        np.testing.assert_allclose(X0[:, k], O.solve_c64(F, B[:, k]), rtol=0, atol=0)
        assert rel_resid(S, X2[:, k], B[:, k]) <= max(rel_resid(S, X0[:, k], B[:, k]), 1e-15) * 1.5


def _emulate_c64(emu, A, merge):
    cp = np.ascontiguousarray(A.colptr - 1)
    rv = np.ascontiguousarray(A.rowval - 1)
    z = np.ascontiguousarray(A.nzval, dtype=np.complex128)
    st = np.zeros(6, np.int64)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    emu.emu_factor_c64(ctypes.c_int64(A.n), P(cp), P(rv), P(z.view(np.float64)), None, ctypes.c_int(merge), P(st))
    n, nl, nu = A.n, int(st[0]), int(st[1])
    out = dict(Lcolptr=np.empty(n + 1, np.int64), Lrowval=np.empty(nl, np.int64), Lnzval=np.empty(nl, np.complex128),
               Ucolptr=np.empty(n + 1, np.int64), Urowval=np.empty(nu, np.int64), Unzval=np.empty(nu, np.complex128),
               p=np.empty(n, np.int64), q=np.empty(n, np.int64))
    emu.emu_get_c64(P(out["Lcolptr"]), P(out["Lrowval"]), P(out["Lnzval"].view(np.float64)), P(out["Ucolptr"]),
                    P(out["Urowval"]), P(out["Unzval"].view(np.float64)), P(out["p"]), P(out["q"]))
    return out, dict(fronts=int(st[2]), nsuper=int(st[3]))


EMU_CASES = [
    ("hermitian-pattern-300", lambda: (lambda S: (S + S.conj().T).tocsc())(sprand_c(300, 8 / 300, seed=11)), 1e-12),
    ("sprand-1200", lambda: sprand_c(1200, 6 / 1200, seed=3), 1e-12),
    # small shift: most pivots leave the diagonal, merged pivot blocks span
    # several supernodes
    ("pivoting-1500", lambda: sprand_c(1500, 5 / 1500, seed=5, shift=0.5), 1e-8),
]


@pytest.mark.parametrize("merge", [1, 0])
@pytest.mark.parametrize("name,make,rtol", EMU_CASES, ids=[c[0] for c in EMU_CASES])
def test_device_algorithm_on_complex_fronts_matches_the_oracle(emu, name, make, rtol, merge):
    A = O.ComplexCSC.from_scipy(make())
    fo = O.multifrontal_lu_c64(A, check=False)
    got, st = _emulate_c64(emu, A, merge)
    assert st["fronts"] < st["nsuper"] if merge else st["fronts"] == st["nsuper"]
    for key in ("Lcolptr", "Lrowval", "Ucolptr", "Urowval", "p", "q"):
        np.testing.assert_array_equal(got[key], getattr(fo, key), err_msg=key)
    nl, _ = column_value_errors(fo.Lcolptr, fo.Lnzval, got["Lnzval"])
    nu, _ = column_value_errors(fo.Ucolptr, fo.Unzval, got["Unzval"])
    assert max(nl, nu) <= rtol, (nl, nu)
    if name.startswith("pivoting"):
        assert np.count_nonzero(fo.p != fo.q) > A.n // 4   # the pivoting is real


@pytest.mark.parametrize("kind", [O.SCALE_NONE, O.SCALE_SUM, O.SCALE_MAX])
def test_library_row_scaling_c64_is_the_oracles(kind):
    # mfgpu_row_scaling_c64 (host code of libmfgpu) against the oracle: bitwise
    from pureumfpack import _lib

    L = _lib.lib()
    S = sprand_c(500, 8 / 500, seed=71)
    A = O.ComplexCSC.from_scipy(S)
    rs = np.empty(A.n)
    z = np.ascontiguousarray(A.nzval, dtype=np.complex128)
    rc = L.mfgpu_row_scaling_c64(A.n, _lib.ptr(np.ascontiguousarray(A.colptr)), _lib.ptr(np.ascontiguousarray(A.rowval)),
                                 _lib.ptr(z.view(np.float64), _lib.f64p), kind, _lib.ptr(rs, _lib.f64p))
    assert rc == 0
    np.testing.assert_array_equal(rs, O.row_scaling_c64(A, kind))
