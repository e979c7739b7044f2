"""One rank of the two-rank sharding test (run as a script by test_shard.py).

Partitions a fixed list of path graphs over the ranks with a CPU stand-in
for the batched GPU entry point (first half / second half of the vertices)
and writes what rank 0 gathered, and the max-over-ranks of a per-rank value,
to the JSON file named on the command line.
"""
import json
import os
import sys
from datetime import timedelta

import numpy as np
import torch.distributed as dist

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from ipdps_2021_graph_coarsening_b200.graphs import CSR  # noqa: E402
from ipdps_2021_graph_coarsening_b200 import shard  # noqa: E402


def path_graph(n):
    deg = np.full(n, 2, np.uint32)
    deg[0] = deg[-1] = 1
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum(deg)
    col = np.empty(int(rp[-1]), np.uint32)
    for i in range(n):
        nb = [j for j in (i - 1, i + 1) if 0 <= j < n]
        col[rp[i]:rp[i + 1]] = nb
    return CSR(rp, col)


def halves(graphs):
    out = []
    for g in graphs:
        part = (np.arange(g.n) >= g.n // 2).astype(np.uint32)
        out.append({"n": g.n, "cut": 1, "part0": int((part == 0).sum()), "rank": dist.get_rank()})
    return out


def main():
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    sizes = [int(s) for s in os.environ["SHARD_SIZES"].split(",")]
    graphs = [path_graph(s) for s in sizes]
    res = shard.partition_sharded(graphs, halves, rank, world, dist)
    mx = shard.max_over_ranks(rank + 1.5, dist)
    if rank == 0:
        with open(sys.argv[1], "w") as f:
            json.dump({"results": res, "max": mx}, f)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
