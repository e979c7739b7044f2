"""Sharding independent graphs over ranks (one process per GPU): the
longest-processing-time assignment, and a two-rank gather over gloo on the
CPU with a stand-in for the per-rank partition call."""
import json
import os
import socket
import subprocess
import sys

import pytest

from ipdps_2021_graph_coarsening_b200.shard import lpt_assign, max_over_ranks

HERE = os.path.dirname(os.path.abspath(__file__))


def test_lpt_assign_is_a_balanced_partition_of_the_indices():
    costs = [5, 1, 9, 3, 3, 8, 2, 7, 7, 1, 4]
    for ranks in (1, 2, 3, 4, 16):
        a = lpt_assign(costs, ranks)
        assert sorted(i for r in a for i in r) == list(range(len(costs)))
        loads = [sum(costs[i] for i in r) for r in a]
        # LPT bound: no rank exceeds the mean load by more than the largest job
        assert max(loads) <= sum(costs) / ranks + max(costs)
        assert a == lpt_assign(costs, ranks)   # every rank computes the same


def test_lpt_assign_order_and_ties():
    assert lpt_assign([4, 4, 4, 4], 2) == [[0, 2], [1, 3]]
    assert lpt_assign([1, 10, 1], 2) == [[1], [0, 2]]
    assert lpt_assign([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        lpt_assign([1], 0)


def test_max_over_ranks_without_a_group():
    assert max_over_ranks(3.5) == 3.5


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gather_every_graph_once(tmp_path):
    sizes = [300, 20, 55, 1000, 7, 64, 64, 2]
    out = tmp_path / "res.json"
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(free_port()), WORLD_SIZE="2",
               SHARD_SIZES=",".join(map(str, sizes)))
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "shard_worker.py"), str(out)],
                              env=dict(env, RANK=str(r))) for r in range(2)]
    rcs = [p.wait(timeout=120) for p in procs]
    assert rcs == [0, 0]
    d = json.loads(out.read_text())
    assert d["max"] == 2.5
    res = d["results"]
    assert [r["n"] for r in res] == sizes
    assert all(r["part0"] == r["n"] // 2 for r in res)
    # the ranks did the shares that the assignment gives them
    costs = [2 * s - 2 for s in sizes]
    a = lpt_assign(costs, 2)
    for rank in range(2):
        assert sorted(i for i, r in enumerate(res) if r["rank"] == rank) == sorted(a[rank])
