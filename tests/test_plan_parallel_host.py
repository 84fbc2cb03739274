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
    return block_diagonal([A for A, _ in M.batched_set(count, seed=0, nrhs=1)])


def block_diagonal(As):
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


def interleave_pairs(A, S, sys_cols):
    """The same factorization with the supernodes of systems 2i and 2i+1
    interleaved: a topological order of the forest that is not a postorder
    (each system keeps its own order; a pair's trees overlap)."""
    ns = S.nsuper
    sst = S.sstart - 1
    sys_of = np.searchsorted(sys_cols, sst[:-1], side="right") - 1
    order = []
    for a in range(0, len(sys_cols) - 1, 2):
        s1 = list(np.flatnonzero(sys_of == a))
        s2 = list(np.flatnonzero(sys_of == a + 1))
        while s1 or s2:
            if s1:
                order.append(s1.pop(0))
            if s2:
                order.append(s2.pop(0))
    assert sorted(order) == list(range(ns)) and order != sorted(order)
    newcol = np.empty(A.n, np.int64)
    sstart, at = [0], 0
    for s in order:
        w = sst[s + 1] - sst[s]
        newcol[sst[s]:sst[s + 1]] = np.arange(at, at + w)
        at += w
        sstart.append(at)
    qf = np.empty(A.n, np.int64)
    qf[newcol] = S.qf - 1
    par0 = S.parent - 1
    parent = np.full(A.n, -1, np.int64)
    parent[newcol] = np.where(par0 >= 0, newcol[np.maximum(par0, 0)], -1)
    upd_ptr, upd_idx = [0], []
    for s in order:
        u = newcol[S.upd_idx[S.upd_ptr[s] - 1:S.upd_ptr[s + 1] - 1] - 1]
        assert np.all(np.diff(u) > 0)
        upd_idx.extend(u.tolist())
        upd_ptr.append(len(upd_idx))

    class Sym:
        pass

    T = Sym()
    T.qf, T.parent = qf + 1, parent + 1
    T.sstart, T.upd_ptr = np.array(sstart) + 1, np.array(upd_ptr) + 1
    T.upd_idx = np.array(upd_idx, np.int64) + 1
    return T


@pytest.mark.parametrize("merge", [1, 0])
def test_interleaved_trees(emu, monkeypatch, merge):
    As = [A for A, _ in M.batched_set(48, seed=1, nrhs=1)]
    sys_cols = np.cumsum([0] + [A.n for A in As])
    B, S = block_diagonal(As)
    T = interleave_pairs(B, S, sys_cols)
    monkeypatch.setenv("MFGPU_HOST_THREADS", "1")
    one = digest(emu, B, T, merge)
    monkeypatch.delenv("MFGPU_HOST_THREADS")
    many = digest(emu, B, T, merge)
    assert "error" not in one and len(one) >= 86, one
    assert one == many, [k for k in one if one[k] != many.get(k)]
