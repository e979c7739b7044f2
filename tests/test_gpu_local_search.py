"""The reference's local search after the split (sgpar.h:2080-2170) on the
device (split.cu k_local_search) against the reference's own serial build
(oracle/_ref) and the oracle: partitions and cuts bit for bit from the same
vector, and through the partition entry points."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import api
from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O

pytestmark = pytest.mark.gpu


def cut_of(g, labels):
    r = np.repeat(np.arange(g.n), np.diff(g.row_ptr).astype(np.int64))
    return int((labels[r] != labels[g.col]).sum()) // 2


CASES = {
    "grid": lambda: G.grid2d(30, 20),
    "holes": lambda: G.grid2d_holes(60, 50, 0.1, 2),
    "er": lambda: G.erdos_renyi(3000, 5.0, seed=3),
    "rmat": lambda: G.rmat(11, seed=2),
    "odd_path": lambda: G.CSR(*path_csr(1001)),
}


def path_csr(n):
    rows = []
    for i in range(n):
        rows.append([j for j in (i - 1, i + 1) if 0 <= j < n])
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    return rp, np.array([j for r in rows for j in r], np.uint32)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("vec", ["random", "spectral"])
def test_compute_partition_local_search_bit_exact(name, vec):
    g = CASES[name]()
    rng = np.random.default_rng(4)
    ev = rng.standard_normal(g.n) if vec == "random" else \
        O.partition_graph(g.row_ptr, g.col, None, rng_state=9)["evec"]
    part, cut = api.compute_partition(ev, g, 2, 0, local_search_alg=1)
    op, oc, _ = O.compute_partition_ls(g.row_ptr, g.col, ev)
    assert np.array_equal(part, op) and cut == oc == cut_of(g, part)
    if O.ref_available("serial"):
        rp, rc = O.ref_compute_partition_ls(g.row_ptr, g.col, ev)
        assert np.array_equal(part, rp) and cut == rc
    # and it does not worsen the split
    _, c0 = api.compute_partition(ev, g, 2, 0, local_search_alg=0)
    assert cut <= c0


@pytest.mark.parametrize("name", ["holes", "rmat"])
def test_partition_with_local_search(partitioner, name):
    g = CASES[name]()
    base = partitioner.partition(g, rng_state=11)
    r = partitioner.partition(g, rng_state=11, local_search_alg=1)
    assert r.edgecut == cut_of(g, r.part) <= base.edgecut
    assert r.part0_size == int((r.part == 0).sum()) and r.level_n == base.level_n
    o = O.partition_graph(g.row_ptr, g.col, None, rng_state=11, local_search_alg=1)
    assert abs(r.edgecut - o["edgecut"]) <= 0.05 * o["edgecut"] + 4


def test_config_local_search_alg():
    g = CASES["er"]()
    cfg = api.Config(local_search_alg=1, num_iter=1)
    part, cut = api.partition_graph(g, cfg, 0, api.PCG32(state=3, inc=1))
    part0, cut0 = api.partition_graph(g, api.Config(num_iter=1), 0, api.PCG32(state=3, inc=1))
    assert cut == cut_of(g, part) <= cut0
