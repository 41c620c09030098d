"""The N > 1 path on the CPU: two gloo ranks split the 64-problem batch by
cost, agree on the slowest rank's time and gather every problem's result on
rank 0 -- the host logic bench.py runs under torchrun (no GPU needed) -- and
solve a batch end to end through solve_sharded, each rank solving its share
with the FP64 oracle standing in for the batched GPU call."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import workloads as W  # noqa: E402
from mps3d_b200.shard import partition_by_cost  # noqa: E402


def test_partition_covers_and_balances():
    costs = [n ** 3 for n in W.batch_sizes(64)]
    for nr in (1, 2, 4, 8):
        parts = partition_by_cost(costs, nr)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in p) for p in parts]
        # within one per cent of a perfect split for this batch (LPT is <= 4/3 in general)
        assert max(loads) <= 1.01 * sum(costs) / nr
    assert partition_by_cost([5.0, 1.0, 1.0], 2) == [[0], [1, 2]]
    with pytest.raises(ValueError):
        partition_by_cost([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, ws):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist

    from mps3d_b200 import workloads as Wk
    from mps3d_b200.shard import barrier, dist_init, dist_max, gather_results, partition_by_cost as part

    w, r, _ = dist_init(timeout_s=60, backend="gloo")
    assert (w, r) == (ws, rank)
    costs = [n ** 3 for n in Wk.batch_sizes(64)]
    mine = part(costs, w)[r]
    # the same partition on every rank, disjoint shares
    every_share = [None] * w
    dist.all_gather_object(every_share, mine)
    assert sorted(i for s in every_share for i in s) == list(range(64))
    t = dist_max(1.5 + r, w)
    assert t == 1.5 + (w - 1)
    local = [{"problem": i, "rank": r, "cells": costs[i]} for i in mine]
    out = gather_results(local, mine, w, r, 64)
    if r == 0:
        assert [o["problem"] for o in out] == list(range(64))
        assert {o["rank"] for o in out} == set(range(w))
    else:
        assert out is None
    barrier(w)
    dist.destroy_process_group()


def test_two_gloo_ranks_share_the_batch():
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(_free_port(), 2), nprocs=2, start_method="spawn", join=True)


def _solve_rank_main(rank, port, ws, sizes):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import numpy as np
    import torch.distributed as dist

    from mps3d_b200 import workloads as Wk
    from mps3d_b200.shard import barrier, dist_init, solve_sharded
    from oracle import oracle as O

    w, r, _ = dist_init(timeout_s=60, backend="gloo")
    probs = Wk.batch_poisson(len(sizes), sizes=tuple(sorted(set(sizes))))

    def solve_share(ps):  # the stand-in of one batched call: the oracle, problem by problem
        out = []
        for p in ps:
            x, hist = O.RowsMG(p, hier=O.HIER_GEOM).solve(O.build_rhs(p), maxit=60, tol=1e-12)
            out.append({"x": x, "rel": float(hist[-1]), "rank": r})
        return out

    res, mine = solve_sharded(probs, solve_share, w, r)
    if r == 0:
        assert len(res) == len(probs) and all(x is not None for x in res)
        assert {x["rank"] for x in res} == set(range(w))
        for p, x in zip(probs, res):  # each gathered solution is its own problem's
            ref, _ = O.RowsMG(p, hier=O.HIER_GEOM).solve(O.build_rhs(p), maxit=60, tol=1e-12)
            assert x["x"].shape == p.shape and x["rel"] <= 1e-12
            assert np.abs(x["x"] - ref).max() <= 1e-12 * np.abs(ref).max()
    else:
        assert res is None
    barrier(w)
    dist.destroy_process_group()


def test_two_gloo_ranks_solve_a_batch_end_to_end():
    import torch.multiprocessing as mp

    mp.start_processes(_solve_rank_main, args=(_free_port(), 2, [5, 7, 9, 7, 5, 9, 9, 5]), nprocs=2,
                       start_method="spawn", join=True)
