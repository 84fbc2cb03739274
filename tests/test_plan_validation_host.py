"""A caller's symbolic analysis is checked before anything is indexed by it.

mfgpu_analyze takes the reference's SymbolicMF arrays (qf, parent, sstart
and the update sets, src/symbolic.jl:203-209) from its caller.  An
inconsistent set (a bad partition, unsorted or out-of-range update rows, a
parent that is not an elimination tree, a symbolic analysis of another
matrix) must be rejected as an argument error by the plan builders on the
host, with merged fronts and with one front per supernode, before a map
reaches the device; the reference itself raises a BoundsError or
ArgumentError for such input.  Run here through tests/plan_emulator.cpp,
which links the library's own plan and symbolic sources.
"""

import ctypes

import numpy as np
import pytest

from pureumfpack import SparseCSC, colamd_order, symbolic_mf
from pureumfpack import matrices as M


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def build(emu, A, arrays, merge):
    """0 = plan built, 1 = rejected as invalid, 2 = another failure."""
    qf, parent, sstart, upd_ptr, upd_idx = (np.ascontiguousarray(a, dtype=np.int64) for a in arrays)
    cp = np.ascontiguousarray(A.colptr - 1)
    rv = np.ascontiguousarray(A.rowval - 1)
    msg = ctypes.create_string_buffer(256)
    rc = emu.emu_build_plan(ctypes.c_int64(A.n), _ptr(cp), _ptr(rv), _ptr(qf), _ptr(parent),
                            ctypes.c_int64(len(sstart) - 1), _ptr(sstart), _ptr(upd_ptr),
                            _ptr(upd_idx) if len(upd_idx) else None, ctypes.c_int(merge), msg, ctypes.c_int64(256))
    return rc, msg.value.decode()


def zero_based(S):
    return [S.qf - 1, S.parent - 1, S.sstart - 1, S.upd_ptr - 1, S.upd_idx - 1]


def _first(cond):
    idx = np.flatnonzero(cond)
    assert len(idx), "the matrix lacks the structure this corruption needs"
    return int(idx[0])


def corrupt(name, arrays, n):
    qf, parent, sstart, upd_ptr, upd_idx = (a.copy() for a in arrays)
    ns = len(sstart) - 1
    nu = np.diff(upd_ptr)
    if name == "partition-short":
        sstart[-1] = n - 1
    elif name == "partition-empty":
        s = _first(np.diff(sstart)[:-1] >= 1)
        sstart[s + 1] = sstart[s]
    elif name == "partition-beyond-n":
        sstart[ns // 2] = n + 7
    elif name == "upd-ptr-start":
        upd_ptr[0] = 1
    elif name == "upd-ptr-decreasing":
        s = _first(nu[:-1] > 0)
        upd_ptr[s + 1] = upd_ptr[s + 2] + 1 if s + 2 <= ns else upd_ptr[s] - 1
    elif name == "upd-row-out-of-range":
        s = _first(nu > 0)
        upd_idx[upd_ptr[s + 1] - 1] = n
    elif name == "upd-row-negative":
        s = _first(nu > 0)
        upd_idx[upd_ptr[s]] = -3
    elif name == "upd-rows-unsorted":
        s = _first(nu > 1)
        p = upd_ptr[s]
        upd_idx[p], upd_idx[p + 1] = upd_idx[p + 1], upd_idx[p]
    elif name == "upd-row-inside-supernode":
        s = _first((nu > 0) & (np.diff(sstart) > 1))
        upd_idx[upd_ptr[s]] = sstart[s]
    elif name == "upd-row-missing-from-parent":
        # drop a row from a parent's update set that one of its children holds
        S_par = parent[sstart[1:] - 1]
        sup_of = np.repeat(np.arange(ns), np.diff(sstart))
        for s in range(ns):
            if S_par[s] < 0:
                continue
            ps = sup_of[S_par[s]]
            pset = upd_idx[upd_ptr[ps]:upd_ptr[ps + 1]]
            child = upd_idx[upd_ptr[s]:upd_ptr[s + 1]]
            common = np.intersect1d(pset, child)
            if len(common):
                drop = upd_ptr[ps] + int(np.searchsorted(pset, common[-1]))
                upd_idx = np.delete(upd_idx, drop)
                upd_ptr[ps + 1:] -= 1
                break
        else:
            raise AssertionError("no child shares an update row with its parent")
    elif name == "parent-out-of-range":
        parent[0] = n
    elif name == "parent-below-self":
        parent[n // 2] = n // 2
    elif name == "parent-negative":
        parent[1] = -2
    elif name == "qf-duplicate":
        qf[1] = qf[0]
    elif name == "qf-out-of-range":
        qf[-1] = n
    elif name == "no-supernodes":
        sstart, upd_ptr, upd_idx = np.array([0]), np.array([0]), np.array([], np.int64)
    else:
        raise KeyError(name)
    return [qf, parent, sstart, upd_ptr, upd_idx]


CORRUPTIONS = ["partition-short", "partition-empty", "partition-beyond-n", "upd-ptr-start", "upd-ptr-decreasing",
               "upd-row-out-of-range", "upd-row-negative", "upd-rows-unsorted", "upd-row-inside-supernode",
               "upd-row-missing-from-parent", "parent-out-of-range", "parent-below-self", "parent-negative",
               "qf-duplicate", "qf-out-of-range", "no-supernodes"]

MATRICES = [
    ("poisson3d-8", lambda: M.poisson3d(8), False),
    ("convdiff-8-colamd", lambda: M.convdiff3d(8), True),
]


@pytest.mark.parametrize("merge", [1, 0])
@pytest.mark.parametrize("mname,make,use_colamd", MATRICES, ids=[m[0] for m in MATRICES])
def test_valid_symbolic_builds(emu, mname, make, use_colamd, merge):
    A = make()
    S = symbolic_mf(A, q=colamd_order(A) if use_colamd else None)
    assert build(emu, A, zero_based(S), merge) == (0, "")
    S = symbolic_mf(A, q=colamd_order(A) if use_colamd else None, relax=True)
    assert build(emu, A, zero_based(S), merge) == (0, "")


@pytest.mark.parametrize("merge", [1, 0])
@pytest.mark.parametrize("what", CORRUPTIONS)
@pytest.mark.parametrize("mname,make,use_colamd", MATRICES, ids=[m[0] for m in MATRICES])
def test_inconsistent_symbolic_is_rejected(emu, mname, make, use_colamd, what, merge):
    A = make()
    S = symbolic_mf(A, q=colamd_order(A) if use_colamd else None)
    rc, msg = build(emu, A, corrupt(what, zero_based(S), A.n), merge)
    assert rc == 1 and msg, (rc, msg)


@pytest.mark.parametrize("merge", [1, 0])
def test_symbolic_of_another_matrix_is_rejected(emu, merge):
    A = M.poisson3d(8)
    n = A.n
    D = SparseCSC.from_coo(np.arange(1, n + 1), np.arange(1, n + 1), np.ones(n), n, n)
    rc, msg = build(emu, A, zero_based(symbolic_mf(D)), merge)
    assert rc == 1 and "symbolic structure" in msg, (rc, msg)
    # the same ordering of a sparser pattern: A has entries outside its fronts
    B = M.poisson2d(int(round(np.sqrt(n))))
    if B.n == n:
        rc, msg = build(emu, A, zero_based(symbolic_mf(B)), merge)
        assert rc == 1, (rc, msg)
