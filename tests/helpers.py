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
    non-cancelled entries).  Columns are the contiguous segments of the
    1-based colptr, reduced with ufunc.reduceat (fast at 10^8 entries)."""
    ref = np.asarray(ref)     # real or complex values; only magnitudes are reduced
    got = np.asarray(got)
    colptr = np.asarray(colptr, dtype=np.int64)
    cnt = np.diff(colptr)
    if ref.size == 0:
        return 0.0, 0.0
    starts = colptr[:-1][cnt > 0] - 1
    aref = np.abs(ref)
    d = np.abs(got - ref)
    colmax = np.maximum.reduceat(aref, starts)
    coln2 = np.add.reduceat(aref * aref, starts)
    errn2 = np.add.reduceat(d * d, starts)
    nz = coln2 > 0
    normwise = float(np.max(np.sqrt(errn2[nz] / coln2[nz]))) if nz.any() else 0.0
    floor = np.repeat(CANCEL_FLOOR * colmax, cnt[cnt > 0])
    big = aref > floor
    entry = float(np.max(d[big] / aref[big])) if big.any() else 0.0
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


def symbolic_pattern(S):
    """The factor pattern that the symbolic analysis alone fixes
    (src/multifrontal.jl:73-104 for the column counts, :278-317 for the
    scatter order), vectorised for 10^8-entry factors.

    Returns a dict of 0-based arrays:
      Lcolptr, Ucolptr (1-based, n + 1);
      Urowval (1-based): column j holds, for every supernode t before j's own
        whose update set contains j (in supernode order), rows c1(t)..c2(t),
        then its own rows c1(s)..j -- no pivot enters U's pattern;
      Lpiv_pos / Lpiv_val: L's pivot-block entries (relabelled rows, 1-based
        values c1+a..c2 after the diagonal) -- pivot-independent because the
        relabelling maps each supernode's pivot rows onto its own columns;
      Lupd_pos / Lupd_val: L's update-set entries as rows of the symbolic
        order (0-based, before the relabelling, which depends on the pivots).
    """
    n = int(S.n)
    ss = np.asarray(S.sstart, np.int64) - 1
    ns = len(ss) - 1
    up = np.asarray(S.upd_ptr, np.int64) - 1
    ui = np.asarray(S.upd_idx, np.int64) - 1
    npv = np.diff(ss)
    nuv = np.diff(up)
    col_s = np.repeat(np.arange(ns), npv)
    cols = np.arange(n, dtype=np.int64)
    c2 = ss[1:][col_s]

    def ranges(lengths):
        """(owner index, position within its range) for consecutive ranges."""
        owner = np.repeat(np.arange(len(lengths), dtype=np.int64), lengths)
        first = np.cumsum(lengths) - lengths
        return owner, np.arange(int(lengths.sum()), dtype=np.int64) - np.repeat(first, lengths)

    # L: column g of supernode s: rows g..c2-1 (pivot block), then upd(s)
    lenpiv = c2 - cols
    lennu = nuv[col_s]
    Lcolptr = np.concatenate([[1], 1 + np.cumsum(lenpiv + lennu)])
    g, w = ranges(lenpiv)
    Lpiv_pos = Lcolptr[g] - 1 + w
    Lpiv_val = g + w + 1
    g, w = ranges(lennu)
    Lupd_pos = Lcolptr[g] - 1 + lenpiv[g] + w
    Lupd_val = ui[up[col_s[g]] + w]
    del g, w
    # U: pairs (t, j) for j in upd(t), grouped by column j in supernode order
    pair_t = np.repeat(np.arange(ns), nuv)
    pair_col = ui
    order = np.argsort(pair_col, kind="stable")
    pt, pc = pair_t[order], pair_col[order]
    plen = npv[pt]
    own = cols - ss[col_s] + 1
    ucount = own + np.bincount(pc, weights=plen, minlength=n).astype(np.int64)
    Ucolptr = np.concatenate([[1], 1 + np.cumsum(ucount)])
    excl = np.cumsum(plen) - plen
    first_of_col = np.searchsorted(pc, pc, side="left")
    in_col = excl - excl[first_of_col]
    Urowval = np.empty(int(Ucolptr[-1] - 1), np.int64)
    e, w = ranges(plen)
    Urowval[Ucolptr[pc[e]] - 1 + in_col[e] + w] = ss[pt[e]] + w + 1
    del e, w
    g, w = ranges(own)
    Urowval[Ucolptr[g] - 1 + (ucount[g] - own[g]) + w] = ss[col_s[g]] + w + 1
    return {"Lcolptr": Lcolptr, "Ucolptr": Ucolptr, "Urowval": Urowval, "Lpiv_pos": Lpiv_pos,
            "Lpiv_val": Lpiv_val, "Lupd_pos": Lupd_pos, "Lupd_val": Lupd_val}


def assert_structure_from_symbolic(S, L, U, p):
    """The factors' pattern against symbolic_pattern(S), and the pivot rows
    of every supernode chosen inside its own pivot block: L's update rows,
    un-relabelled through the row permutation that p = qf[prow] implies,
    must be the symbolic update sets exactly."""
    E = symbolic_pattern(S)
    np.testing.assert_array_equal(L.colptr, E["Lcolptr"])
    np.testing.assert_array_equal(U.colptr, E["Ucolptr"])
    np.testing.assert_array_equal(U.rowval, E["Urowval"])
    Lr = np.asarray(L.rowval, np.int64)
    np.testing.assert_array_equal(Lr[E["Lpiv_pos"]], E["Lpiv_val"])
    qf = np.asarray(S.qf, np.int64) - 1
    qfinv = np.empty_like(qf)
    qfinv[qf] = np.arange(len(qf))
    prow = qfinv[np.asarray(p, np.int64) - 1]          # p = qf[prow]
    ss = np.asarray(S.sstart, np.int64) - 1
    block = np.repeat(np.arange(len(ss) - 1), np.diff(ss))
    np.testing.assert_array_equal(block[prow], block)   # pivots stay in their block
    np.testing.assert_array_equal(prow[Lr[E["Lupd_pos"]] - 1], E["Lupd_val"])
