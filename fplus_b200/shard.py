"""Sharding independent factorizations across GPUs (one process per GPU).

The batch form's units are independent pencils (one per Dedalus subproblem, or shifts sigma_k of one pattern): they are
partitioned across ranks by predicted cost with the greedy longest-processing-time rule (Graham 1969: each job, largest
first, goes to the least-loaded rank; the makespan is within 4/3 of the optimum).  Every rank computes the same partition
from the same costs, so no data moves between GPUs: each rank factors and solves its own share on its own GPU, and only
the per-rank results (status, timing) are gathered at the end (torch.distributed all_gather_object over NCCL or gloo).
"""
from __future__ import annotations

import heapq


def lpt_partition(costs, nparts):
    """Indices of `costs` split into `nparts` lists by the LPT rule; ties go to the lower rank.  Within each list the
    jobs come largest first (the order in which a rank should start them)."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(nparts)]
    parts = [[] for _ in range(nparts)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return parts


def pencil_cost(n, nnz, flops=None):
    """The cost proxy of one factorization: the front structure's multiply-adds when known, else n * nnz."""
    return float(flops) if flops is not None else float(n) * float(nnz)


def gather_results(obj):
    """Every rank's `obj`, in rank order (a list of length 1 without an initialised process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
