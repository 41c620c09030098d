"""Work across ranks (one process per GPU): independent solves, no collective
on the data path.

The single-grid solve does not shard (the whole grid lives on one GPU; the
reference's MPI halo exchange, par_decompose.f90:122-296, becomes on-device
ghost layers), so N GPUs run N replicas.  A batch of independent problems
is split by size: greedy longest-processing-time assignment with cost
proportional to the cell count, each rank solving its share with one batched
call.  Host-side collectives only: the max over ranks of the device time
and a gather of the per-problem results on rank 0.
"""
from __future__ import annotations

import datetime
import os
from typing import List, Sequence


def dist_init(timeout_s: int = 600, backend: str = None):
    """(world size, rank, local rank) from the torchrun environment; creates
    the process group (NCCL with a GPU, gloo without, unless ``backend`` is
    given) when world size > 1."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist

        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    """Max of x over the ranks (device timings are reported as the slowest rank)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if (torch.cuda.is_available() and dist.get_backend() == "nccl") else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def partition_by_cost(costs: Sequence[float], nranks: int) -> List[List[int]]:
    """Problem indices per rank: largest first, each to the least-loaded rank
    (ties to the lower rank), indices kept in ascending order per rank."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * nranks
    parts: List[List[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def gather_results(local: list, indices: Sequence[int], ws: int, rank: int, total: int):
    """Rank 0 gets the per-problem results of every rank in problem order
    (None elsewhere)."""
    if ws == 1:
        out = [None] * total
        for i, r in zip(indices, local):
            out[i] = r
        return out
    import torch.distributed as dist

    pairs = list(zip(indices, local))
    got = [None] * ws if rank == 0 else None
    dist.gather_object(pairs, got, dst=0)
    if rank != 0:
        return None
    out = [None] * total
    for part in got:
        for i, r in part:
            out[i] = r
    return out


def solve_sharded(problems: Sequence, solve_share, ws: int, rank: int, cost=None):
    """Independent problems across ranks: each rank solves its cost-balanced
    share (``solve_share(list of problems) -> list of results``, one per
    problem, e.g. one batched GPU call) and rank 0 receives every result in
    problem order (None on the other ranks).  Returns (results, this rank's
    problem indices)."""
    cost = cost or (lambda p: p.lx * p.ly * p.lz)
    mine = partition_by_cost([cost(p) for p in problems], ws)[rank]
    local = list(solve_share([problems[i] for i in mine])) if mine else []
    if len(local) != len(mine):
        raise RuntimeError("solve_share returned %d results for %d problems" % (len(local), len(mine)))
    return gather_results(local, mine, ws, rank, len(problems)), mine
