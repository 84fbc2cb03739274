"""The plan's parallel host loops give the sequential plan.

The plan builder fills its per-column arrays range by range over the trees
of the supernode forest, and its per-column and per-supernode maps, on all
host cores.  Every field of the plan must equal the plan built on one
thread (MFGPU_HOST_THREADS=1; the ranges are then also cut differently), for
a forest of many trees (a batch of independent systems) and for single
matrices, with merged fronts and with one front per supernode.
"""

import ctypes

import numpy as np
import pytest

from pureumfpack import colamd_order, symbolic_mf
from pureumfpack import matrices as M
from pureumfpack.api import symbolic_batch
from pureumfpack.sparse import SparseCSC


def digest(emu, A, S, merge):
    arrs = [np.ascontiguousarray(a, dtype=np.int64)
            for a in (A.colptr - 1, A.rowval - 1, S.qf - 1, S.parent - 1, S.sstart - 1, S.upd_ptr - 1, S.upd_idx - 1)]
    p = [a.ctypes.data_as(ctypes.c_void_p) for a in arrs]
    emu.emu_plan_digest.restype = ctypes.c_char_p
    d = emu.emu_plan_digest(ctypes.c_int64(A.n), p[0], p[1], p[2], p[3], ctypes.c_int64(len(arrs[4]) - 1), p[4],
                            p[5], p[6], ctypes.c_int(merge))
    return dict(kv.split("=") for kv in d.decode().strip(";").split(";"))


def batch(count):
    As = [A for A, _ in M.batched_set(count, seed=0, nrhs=1)]
    offs = np.cumsum([0] + [A.n for A in As])
    nzo = np.cumsum([0] + [A.nnz() for A in As])
    cp = np.concatenate([[1]] + [A.colptr[1:] + z for A, z in zip(As, nzo[:-1])])
    rv = np.concatenate([A.rowval + o for A, o in zip(As, offs[:-1])])
    B = SparseCSC(int(offs[-1]), int(offs[-1]), cp, rv, np.ones(len(rv)))
    return B, symbolic_batch(As, "amd")


def single(A, col=False):
    return A, symbolic_mf(A, q=colamd_order(A) if col else None)


CASES = [
    ("batch-160", lambda: batch(160)),
    ("poisson3d-20", lambda: single(M.poisson3d(20))),
    ("convdiff-14-colamd", lambda: single(M.convdiff3d(14), col=True)),
    ("random-3000", lambda: single(M.random_unsym(3000, 5, 1.0, seed=3))),
]


@pytest.mark.parametrize("merge", [1, 0])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_parallel_plan_equals_the_sequential_one(emu, monkeypatch, name, make, merge):
    A, S = make()
    monkeypatch.setenv("MFGPU_HOST_THREADS", "1")
    one = digest(emu, A, S, merge)
    monkeypatch.delenv("MFGPU_HOST_THREADS")
    many = digest(emu, A, S, merge)
    assert len(one) >= 86   # every Plan field
    assert one == many, [k for k in one if one[k] != many.get(k)]
