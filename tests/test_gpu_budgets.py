"""Give-up paths of the coarsening constructions.

Each device construction has a round or iteration bound from its progress
argument -- the HEC map rounds 2n + 4 (hec.cu), the matching rounds n + 4 and
the MIS-2 / GOSH independent-set iterations 4n + 16 (coarsen_alt.cu) -- after
which it returns SGP_B200_ERR_BUDGET with a message instead of running on.
The bounds are never reached by correct code, so SGPB_ROUND_CAP (a test hook
that can only lower a bound) makes the path reachable here.  Each test checks
the error code and message, then that the same context serves the next call
with the natural bound and that call equals the oracle.  No kernel faults or
hangs on this path: the cooperative kernels leave their round loop together
and report the error through their result words.
"""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.fixture
def tiny_cap(monkeypatch):
    monkeypatch.setenv("SGPB_ROUND_CAP", "1")
    yield monkeypatch


def test_hec_map_round_budget(partitioner, tiny_cap):
    g = G.rmat(12, seed=4)
    seed = 0x5EED
    hn_o = O.hec_heavy(g.row_ptr, g.col, None, True, seed)
    vc_o, nc_o, rounds_o = O.hec_map(hn_o, seed)
    assert rounds_o > 1   # the graph needs more rounds than the cap allows
    with pytest.raises(L.SgparError) as ei:
        partitioner.hec(dev(g.row_ptr), dev(g.col), None, True, seed)
    assert ei.value.code == L.ERR_BUDGET
    assert "HEC map construction exceeded 1 rounds" in L.last_error()
    tiny_cap.delenv("SGPB_ROUND_CAP")
    hn, vc, nc, rounds = partitioner.hec(dev(g.row_ptr), dev(g.col), None, True, seed)
    assert nc == nc_o and rounds == rounds_o
    assert np.array_equal(host(vc), vc_o) and np.array_equal(host(hn), hn_o)


def test_match_round_budget(partitioner, tiny_cap):
    g = G.grid2d(80, 60)
    seed = 0xC0FFEE
    vc_o, nc_o, rounds_o = O.match_map(g.row_ptr, g.col, None, True, seed)
    assert rounds_o > 1
    with pytest.raises(L.SgparError) as ei:
        partitioner.coarsen_map(dev(g.row_ptr), dev(g.col), None, L.COARSEN_MATCH, True, seed)
    assert ei.value.code == L.ERR_BUDGET
    assert "matching exceeded 1 rounds" in L.last_error()
    tiny_cap.delenv("SGPB_ROUND_CAP")
    vc, nc, rounds = partitioner.coarsen_map(dev(g.row_ptr), dev(g.col), None, L.COARSEN_MATCH, True, seed)
    assert nc == nc_o and rounds == rounds_o and np.array_equal(host(vc), vc_o)


@pytest.mark.parametrize("coarsener", [L.COARSEN_MIS2, L.COARSEN_GOSH])
def test_independent_set_iteration_budget(partitioner, tiny_cap, coarsener):
    g = G.grid2d_holes(90, 70, 0.1, 3)
    seed = 0xABC
    vc_o, nc_o, its_o = O.set_map(g.row_ptr, g.col, coarsener == L.COARSEN_GOSH, seed)
    assert its_o > 2   # iterations 0 and 1 are within a cap of 1
    with pytest.raises(L.SgparError) as ei:
        partitioner.coarsen_map(dev(g.row_ptr), dev(g.col), None, coarsener, False, seed)
    assert ei.value.code == L.ERR_BUDGET
    assert "independent-set iterations exceeded 1" in L.last_error()
    tiny_cap.delenv("SGPB_ROUND_CAP")
    vc, nc, its = partitioner.coarsen_map(dev(g.row_ptr), dev(g.col), None, coarsener, False, seed)
    assert nc == nc_o and its == its_o and np.array_equal(host(vc), vc_o)


def test_partition_reports_budget_and_recovers(partitioner, tiny_cap):
    """The error surfaces through the partition entry point, which releases
    its work memory; the next partition on the same context is unaffected."""
    g = G.grid2d(64, 48)
    with pytest.raises(L.SgparError) as ei:
        partitioner.partition(g, rng_state=21)
    assert ei.value.code == L.ERR_BUDGET
    tiny_cap.delenv("SGPB_ROUND_CAP")
    r = partitioner.partition(g, rng_state=21)
    o = O.partition_graph(g.row_ptr, g.col, None, rng_state=21)
    assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
    assert r.edgecut == O.edge_cut(g.row_ptr, g.col, r.part)
