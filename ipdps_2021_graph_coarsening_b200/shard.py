"""Several GPUs, one process each: sharding of independent graphs.

A single graph's partition does not shard (a row partition of the power
iteration would need a halo exchange per iteration); a batch of graphs does.
The graphs are dealt to the ranks largest first, each to the rank with the
least work so far (longest-processing-time-first on the directed entry
count), every rank partitions its share with the batched entry point, and
rank 0 gathers the results.  There is no collective on the data path: the
only exchanges are the final gather and the max-over-ranks of timings.
"""
from __future__ import annotations

from typing import Callable, Sequence


def lpt_assign(costs: Sequence[int], nranks: int) -> list[list[int]]:
    """Indices of ``costs`` per rank: descending cost (ties by index), each
    to the least-loaded rank (ties by rank).  Deterministic, so every rank
    computes the same assignment without communicating."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    load = [0] * nranks
    out: list[list[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(costs[i])
    return out


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """The maximum of ``x`` over all ranks (``x`` itself without a process
    group): the job's time is its slowest rank's."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def partition_sharded(graphs: Sequence, partition_many: Callable[[list], list], rank: int, world: int,
                      dist=None) -> list | None:
    """Partition ``graphs`` over ``world`` ranks.  ``partition_many(list of
    graphs) -> list of results`` runs one rank's share (e.g. a bound
    ``Partitioner.partition_batch``).  Returns, on rank 0, the results in
    the order of ``graphs``; ``None`` on the other ranks."""
    costs = [int(g.m_directed) for g in graphs]
    share = lpt_assign(costs, world)[rank]
    mine = partition_many([graphs[i] for i in share]) if share else []
    local = list(zip(share, mine))
    if dist is None or world == 1:
        gathered = [local]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
    if rank != 0:
        return None
    out = [None] * len(graphs)
    for part in gathered:
        for i, r in part:
            if out[i] is not None:
                raise RuntimeError(f"graph {i} partitioned twice")
            out[i] = r
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise RuntimeError(f"graphs {missing[:8]} were not partitioned")
    return out
