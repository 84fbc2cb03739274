"""The factorization's launch list, executed on the CPU launch by launch.

tests/plan_emulator.cpp runs the plan's launches in order -- small fronts,
column assembly, 64-column panels (speculative, then the pivoting rerun when
a speculative panel meets a larger candidate), the panel triangular solves
and every GEMM task of the blocked updates -- and compares every front with
a plain right-looking elimination of the same fronts.  Each entry receives
the same updates in the same order either way, so a complete and correctly
ordered schedule reproduces it exactly; a missing, duplicated or early task
shows up as a difference."""

import ctypes

import numpy as np
import pytest

from pureumfpack import colamd_order
from pureumfpack import matrices as M


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


CASES = [
    ("poisson3d-16", lambda: M.poisson3d(16), False, False),
    ("convdiff-12-colamd", lambda: M.convdiff3d(12), True, False),
    ("pivoting-2500", lambda: M.random_unsym(2500, 5, 1.0, seed=7), False, True),
    ("pivoting-2500-colamd", lambda: M.random_unsym(2500, 5, 1.0, seed=7), True, True),
]


@pytest.mark.parametrize("merge", [1, 0], ids=["merged", "single"])
@pytest.mark.parametrize("name,make,use_colamd,pivots", CASES, ids=[c[0] for c in CASES])
def test_launch_list_reproduces_elimination(emu, name, make, use_colamd, pivots, merge):
    A = make()
    q = colamd_order(A) if use_colamd else None
    cp = np.ascontiguousarray(A.colptr - 1)
    rv = np.ascontiguousarray(A.rowval - 1)
    qq = None if q is None else np.ascontiguousarray(np.asarray(q, dtype=np.int64) - 1)
    out = np.zeros(4)
    emu.emu_check_launches(ctypes.c_int64(A.n), _ptr(cp), _ptr(rv), _ptr(A.nzval), None if qq is None else _ptr(qq),
                           ctypes.c_int(merge), _ptr(out))
    worst, mismatches, reran, _ = out
    assert worst == 0.0 and mismatches == 0
    assert reran == (1.0 if pivots else 0.0)   # the pivoting matrices exercise the rerun's launch list
