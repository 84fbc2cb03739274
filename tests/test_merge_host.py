"""Merged fronts, host side: the plan's maps checked on the CPU.

tests/plan_emulator.cpp runs the device factorization's semantics over the
library's own Plan (assembly maps, pivot segments, CSC scatter maps), with
merged fronts and with one front per supernode.  Both must reproduce the
oracle's multifrontal_lu exactly in structure and pivot sequence
(src/multifrontal.jl:247-263: pivots only among a supernode's own pivot
rows) and to rounding in value.  The strongly pivoting matrices make the
pivot segments matter: without them the merged fronts would choose pivots
from other supernodes' rows.
"""

import ctypes

import numpy as np
import pytest

from helpers import column_value_errors
from oracle import oracle as O
from pureumfpack import colamd_order
from pureumfpack import matrices as M


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def emulate(lib, A, q, merge):
    cp = np.ascontiguousarray(A.colptr - 1)
    rv = np.ascontiguousarray(A.rowval - 1)
    qq = None if q is None else np.ascontiguousarray(np.asarray(q, dtype=np.int64) - 1)
    st = np.zeros(6, np.int64)
    lib.emu_factor(ctypes.c_int64(A.n), _ptr(cp), _ptr(rv), _ptr(A.nzval), None if qq is None else _ptr(qq),
                   ctypes.c_int(merge), _ptr(st))
    n, nl, nu = A.n, int(st[0]), int(st[1])
    out = dict(Lcolptr=np.empty(n + 1, np.int64), Lrowval=np.empty(nl, np.int64), Lnzval=np.empty(nl),
               Ucolptr=np.empty(n + 1, np.int64), Urowval=np.empty(nu, np.int64), Unzval=np.empty(nu),
               p=np.empty(n, np.int64), q=np.empty(n, np.int64))
    lib.emu_get(*[_ptr(a) for a in out.values()])
    return out, dict(fronts=int(st[2]), nsuper=int(st[3]), max_front=int(st[4]), max_pivots=int(st[5]))


CASES = [
    ("poisson2d-30", lambda: M.poisson2d(30), False, 1e-12),
    ("poisson3d-10", lambda: M.poisson3d(10), False, 1e-12),
    ("convdiff-12-colamd", lambda: M.convdiff3d(12), True, 1e-12),
    ("pivoting-400-colamd", lambda: M.random_unsym(400, 5, 0.3, seed=1), True, 1e-8),
    ("pivoting-800-amd", lambda: M.random_unsym(800, 5, 0.5, seed=2), False, 1e-8),
    ("pivoting-1500-colamd", lambda: M.random_unsym(1500, 5, 1.0, seed=3), True, 1e-8),
]


@pytest.mark.parametrize("name,make,use_colamd,rtol", CASES, ids=[c[0] for c in CASES])
def test_merged_plan_reproduces_oracle(emu, name, make, use_colamd, rtol):
    A = make()
    q = colamd_order(A) if use_colamd else None
    fo = O.multifrontal_lu(A, q=q, check=False)
    merged, sm = emulate(emu, A, q, 1)
    single, su = emulate(emu, A, q, 0)
    assert sm["fronts"] < su["fronts"] == su["nsuper"] == sm["nsuper"]
    for got in (merged, single):
        for key in ("Lcolptr", "Lrowval", "Ucolptr", "Urowval", "p", "q"):
            np.testing.assert_array_equal(got[key], getattr(fo, key), err_msg=key)
        nl, _ = column_value_errors(fo.Lcolptr, fo.Lnzval, got["Lnzval"])
        nu, _ = column_value_errors(fo.Ucolptr, fo.Unzval, got["Unzval"])
        assert max(nl, nu) <= rtol
