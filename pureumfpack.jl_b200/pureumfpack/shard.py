"""Sharding independent systems across GPUs (one process per GPU).

A batch of independent systems needs no exchange between GPUs: every rank
factors and solves its own share and keeps its factors, so the multi-GPU
path has no device collective.  The split balances the predicted numeric
work of each system, taken from the host symbolic pass with the per-
supernode flop count of the multifrontal elimination
(src/multifrontal.jl:247-268: getrf of the np x np pivot block, the two
triangular solves and the Schur update):
    flops(s) = 2/3 np^3 + 2 np^2 nu + 2 np nu^2,  nf = np + nu.
"""

from __future__ import annotations

import heapq

import numpy as np

from .api import amd_order_sym, colamd_order, symbolic_mf


def supernode_flops(S) -> np.ndarray:
    """Numeric flops of every supernode of a SymbolicMF."""
    np_ = np.diff(S.sstart).astype(np.float64)
    nu = np.diff(S.upd_ptr).astype(np.float64)
    return 2.0 / 3.0 * np_**3 + 2.0 * np_**2 * nu + 2.0 * np_ * nu**2


def system_cost(A, ordering: str = "amd") -> float:
    """Predicted factorization flops of one system (host symbolic only)."""
    q = amd_order_sym(A) if ordering == "amd" else colamd_order(A)
    return float(supernode_flops(symbolic_mf(A, q=q)).sum())


def partition_by_cost(costs, nranks: int) -> list[list[int]]:
    """Split systems into nranks shares of nearly equal total cost: largest
    system first onto the least-loaded rank (ties to the lower rank), each
    share listed in ascending system order.  Deterministic, so every rank
    computes the same split without communication."""
    if nranks < 1:
        raise ValueError("nranks must be positive")
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(nranks)]
    shares: list[list[int]] = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shares]


def share_of(costs, rank: int, world: int) -> list[int]:
    return partition_by_cost(costs, world)[rank]
