"""Host side of the batched path: the block-diagonal forest and the split
of independent systems across ranks (CPU only).

A batch is analyzed as one block-diagonal matrix ordered system by system;
the symbolic pass (src/symbolic.jl:15-226) of that matrix must reproduce
every system's own analysis, offset by the system's first column, so that
each system's factors are exactly its own.  Across GPUs the systems are
split by predicted work with no exchange between ranks; the two-rank test
runs that split over gloo with the oracle standing in for each rank's GPU.
"""

import os

import numpy as np
import pytest

from oracle import oracle as O
from pureumfpack import SparseCSC, amd_order_sym, colamd_order, symbolic_mf
from pureumfpack import matrices as M
from pureumfpack.shard import partition_by_cost, supernode_flops, system_cost


def _batch(count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for t in range(count):
        A = M.poisson2d(int(rng.integers(4, 20))) if t % 3 else M.poisson3d(int(rng.integers(3, 8)))
        out.append(A.add_diagonal(float(rng.random())))
    return out


def _block_diag(As):
    offs = np.cumsum([0] + [A.n for A in As])
    I = np.concatenate([A.rowval + o for A, o in zip(As, offs)])
    J = np.concatenate([A.colind() + 1 + o for A, o in zip(As, offs)])
    V = np.concatenate([A.nzval for A in As])
    return SparseCSC.from_coo(I, J, V, offs[-1], offs[-1]), offs


@pytest.mark.parametrize("ordering", ["amd", "colamd"])
def test_forest_symbolic_equals_per_system(ordering):
    As = _batch(10, seed=1) + [M.convdiff3d(4), M.random_unsym(80, 4, 10.0, seed=4)]
    order = amd_order_sym if ordering == "amd" else colamd_order
    Abd, offs = _block_diag(As)
    S = symbolic_mf(Abd, q=np.concatenate([order(A) + o for A, o in zip(As, offs)]))
    ss = 0
    for A, o in zip(As, offs):
        Si = symbolic_mf(A, q=order(A))
        np.testing.assert_array_equal(S.qf[o:o + A.n], Si.qf + o)
        np.testing.assert_array_equal(S.sstart[ss:ss + Si.nsuper + 1], Si.sstart + o)
        for s in range(1, Si.nsuper + 1):
            np.testing.assert_array_equal(S.update_set(ss + s), Si.update_set(s) + o)
        ss += Si.nsuper
    assert ss == S.nsuper
    # the work of the batch is the sum of the systems' work
    total = supernode_flops(S).sum()
    assert total == pytest.approx(sum(system_cost(A, ordering) for A in As), rel=1e-12)


@pytest.mark.parametrize("ordering", ["amd", "colamd"])
def test_parallel_batch_symbolic_equals_block_diagonal(ordering):
    """symbolic_batch (every system ordered and analysed on its own thread,
    then concatenated) is field for field the block-diagonal analysis."""
    from pureumfpack.api import symbolic_batch

    As = _batch(40, seed=5) + [M.convdiff3d(5), M.random_unsym(120, 4, 10.0, seed=2)]
    order = amd_order_sym if ordering == "amd" else colamd_order
    Abd, offs = _block_diag(As)
    S = symbolic_mf(Abd, q=np.concatenate([order(A) + o for A, o in zip(As, offs)]))
    P = symbolic_batch(As, ordering)
    for f in ("qf", "parent", "colcount", "sstart", "upd_ptr", "upd_idx", "child_ptr", "child_idx"):
        np.testing.assert_array_equal(getattr(P, f), getattr(S, f), err_msg=f)


def test_partition_covers_and_balances():
    rng = np.random.default_rng(3)
    costs = rng.pareto(1.5, 300) + 1.0
    for world in (1, 2, 3, 8):
        shares = partition_by_cost(costs, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        loads = [costs[s].sum() for s in shares]
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9
        assert shares == partition_by_cost(costs, world)   # deterministic
    assert partition_by_cost([5.0, 1.0], 4)[2:] == [[], []]


def _rank_main(rank, world, port, out_dir):
    import pickle

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        As = _batch(12, seed=7)
        rng = np.random.default_rng(11)
        Bs = [rng.standard_normal((A.n, 2)) for A in As]
        costs = [system_cost(A) for A in As]
        mine = partition_by_cost(costs, world)[rank]
        # each rank solves only its share (the oracle stands in for its GPU)
        local = {i: O.solve(O.splu(As[i]), Bs[i], refine=1) for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
        if rank == 0:
            with open(os.path.join(out_dir, "result.pkl"), "wb") as f:
                pickle.dump({"shares": [sorted(g) for g in gathered], "x": {k: v for g in gathered for k, v in g.items()}}, f)
    finally:
        dist.destroy_process_group()


def test_two_rank_split_over_gloo(tmp_path):
    import pickle
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = pickle.load(open(tmp_path / "result.pkl", "rb"))
    As = _batch(12, seed=7)
    rng = np.random.default_rng(11)
    Bs = [rng.standard_normal((A.n, 2)) for A in As]
    assert sorted(i for s in res["shares"] for i in s) == list(range(12))
    assert all(res["shares"])                     # both ranks got work
    for i, A in enumerate(As):
        xo = O.solve(O.splu(A), Bs[i], refine=1)
        np.testing.assert_array_equal(res["x"][i], xo)
