"""Multi-GPU host logic: one process per GPU, independent work per rank.

The single-system path does not shard (it would need the spatial
decomposition and halo exchange the reference has only as a host-staged MPI
scaffold), so N GPUs run N independent replicas.  The batched-replica
workload shards naturally: whole replicas are assigned to ranks, balanced by
atom count, and no data crosses ranks during the run.  Timings are device
times reduced as the maximum over ranks.
"""
from __future__ import annotations

import heapq


def lpt_partition(sizes, nparts: int) -> list:
    """Longest-processing-time assignment of items (by size) to nparts bins:
    largest first, each to the currently lightest bin (ties: lowest bin).
    Returns a list of index lists, each in ascending item order."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    heap = [(0, b) for b in range(nparts)]
    bins = [[] for _ in range(nparts)]
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    for i in order:
        load, b = heapq.heappop(heap)
        bins[b].append(i)
        heapq.heappush(heap, (load + sizes[i], b))
    return [sorted(b) for b in bins]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank value over the process group (the value itself
    without one)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """Sum of a per-rank value over the process group."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_by_replica(local_values, mine, nrep: int, dist=None) -> list:
    """Per-replica results of every rank, back in replica order: rank r
    holds local_values[k] for replica mine[k] (its LPT shard); returns the
    list of all nrep results (one all_gather_object of the (index, value)
    pairs; the local list itself without a process group)."""
    pairs = list(zip([int(i) for i in mine], local_values))
    if dist is not None:
        allp = [None] * dist.get_world_size()
        dist.all_gather_object(allp, pairs)
        pairs = [pv for part in allp for pv in part]
    out = [None] * int(nrep)
    for i, v in pairs:
        if out[i] is not None:
            raise ValueError(f"replica {i} reported twice")
        out[i] = v
    if any(v is None for v in out):
        raise ValueError("a replica is missing from the shards")
    return out

