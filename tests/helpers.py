"""Comparison helpers for the parity tests (GPU factors against the oracle)."""

from __future__ import annotations

import numpy as np

# Factor values: the GPU and the oracle evaluate the same elimination with
# different (but both backward-stable) operation orders, so entries agree to
# rounding.  Columnwise normwise agreement is required to 1e-12; entry-wise
# agreement to 1e-12 relative is required on every entry that is not the
# product of cancellation, i.e. |ref| > 1e-6 * max|column|.  (Entries far
# below their column's scale carry the absolute rounding error of the large
# terms that cancelled into them; the normwise bound covers them.)
VALUE_RTOL = 1e-12
CANCEL_FLOOR = 1e-6


def column_value_errors(colptr, ref, got):
    """(max normwise column error, max entry-wise relative error on
    non-cancelled entries)."""
    ref = np.asarray(ref)
    got = np.asarray(got)
    n = len(colptr) - 1
    d = np.abs(got - ref)
    col = np.repeat(np.arange(n), np.diff(colptr))
    colmax = np.zeros(n)
    np.maximum.at(colmax, col, np.abs(ref))
    coln2 = np.zeros(n)
    np.add.at(coln2, col, np.abs(ref) ** 2)
    errn2 = np.zeros(n)
    np.add.at(errn2, col, d * d)
    nz = coln2 > 0
    normwise = float(np.max(np.sqrt(errn2[nz] / coln2[nz]))) if nz.any() else 0.0
    big = np.abs(ref) > CANCEL_FLOOR * colmax[col]
    entry = float(np.max(d[big] / np.abs(ref[big]))) if big.any() else 0.0
    return normwise, entry


def assert_same_structure(fo, L, U, p, q, pinv):
    np.testing.assert_array_equal(L.colptr, fo.Lcolptr)
    np.testing.assert_array_equal(U.colptr, fo.Ucolptr)
    np.testing.assert_array_equal(L.rowval, fo.Lrowval)
    np.testing.assert_array_equal(U.rowval, fo.Urowval)
    np.testing.assert_array_equal(p, fo.p)
    np.testing.assert_array_equal(q, fo.q)
    np.testing.assert_array_equal(pinv, fo.pinv)


def assert_close_values(fo, L, U, rtol=VALUE_RTOL, entry_rtol=None):
    """Normwise per column within rtol; entry-wise within entry_rtol (default
    rtol).  Matrices with element growth rho amplify rounding differences of
    the two operation orders by about rho, so their entry-wise bound is
    raised while the normwise bound stays."""
    entry_rtol = rtol if entry_rtol is None else entry_rtol
    nl, el = column_value_errors(fo.Lcolptr, fo.Lnzval, L.nzval)
    nu, eu = column_value_errors(fo.Ucolptr, fo.Unzval, U.nzval)
    assert nl <= rtol and nu <= rtol, f"normwise column error L {nl:.2e} U {nu:.2e}"
    assert el <= entry_rtol and eu <= entry_rtol, f"entry-wise error L {el:.2e} U {eu:.2e}"
    return max(nl, nu), max(el, eu)


def reconstruction_error(A, L, U, p, q, Rs=None):
    """||(Rs.*A)[p,q] - L U||_F / max(1, ||A||_F) (test/multifrontal_test.jl:37-38)."""
    import scipy.sparse as sp

    S = A.to_scipy()
    if Rs is not None:
        S = sp.diags(Rs) @ S
    Ap = S.tocsr()[p - 1][:, q - 1]
    R = (Ap - L.to_scipy() @ U.to_scipy()).toarray()
    return np.linalg.norm(R) / max(1.0, sp.linalg.norm(A.to_scipy()))


def backward_error(A, x, b):
    """Normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf), per column (max)."""
    S = A.to_scipy()
    X = x.reshape(len(x), -1)
    B = b.reshape(len(b), -1)
    r = B - S @ X
    an = np.max(np.asarray(abs(S).sum(axis=1)).ravel())
    eta = np.max(np.abs(r), axis=0) / (an * np.max(np.abs(X), axis=0) + np.max(np.abs(B), axis=0))
    return float(np.max(eta))
