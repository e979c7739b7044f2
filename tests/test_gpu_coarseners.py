"""The alternative coarseners on the device (coarsen_alt.cu) against the
oracle's restatement of the same rules (oracle/sgpar_oracle.c): mappings bit
for bit, then the whole path with each coarsener -- hierarchy sizes and rng
advance exactly, the cut within the FP64 tolerance of the other parity tests --
and the sgpar.h config path reading coarsening_alg's bits."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import api
from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def graph_cases():
    return {
        "grid": G.grid2d(120, 90),
        "holes": G.grid2d_holes(150, 120, 0.12, 5),
        "rmat14": G.rmat(14, seed=3),
        "chunglu_w": G.chung_lu(40000, wmax=100, seed=4),
        "er": G.erdos_renyi(30000, 5.0, seed=6),
    }


CASES = graph_cases()


def dev(g):
    rp = torch.from_numpy(g.row_ptr.view(np.int32)).cuda()
    col = torch.from_numpy(g.col.view(np.int32)).cuda()
    w = None if g.w is None else torch.from_numpy(g.w.astype(np.uint32).view(np.int32)).cuda()
    return rp, col, w


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("random_level", [True, False])
def test_match_map_bit_exact(partitioner, name, random_level):
    g = CASES[name]
    rp, col, w = dev(g)
    seed = 0xC0FFEE1234
    vc, nc, rounds = partitioner.coarsen_map(rp, col, w, L.COARSEN_MATCH, random_level, seed)
    ovc, onc, orounds = O.match_map(g.row_ptr, g.col, g.w, random_level, seed)
    assert nc == onc and rounds == orounds
    assert np.array_equal(vc.cpu().numpy().view(np.uint32), ovc)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("coarsener", [L.COARSEN_MIS2, L.COARSEN_GOSH])
def test_set_map_bit_exact(partitioner, name, coarsener):
    g = CASES[name]
    rp, col, _ = dev(g)
    seed = 0xABCDEF987
    vc, nc, its = partitioner.coarsen_map(rp, col, None, coarsener, False, seed)
    ovc, onc, oits = O.set_map(g.row_ptr, g.col, coarsener == L.COARSEN_GOSH, seed)
    assert nc == onc and its == oits
    assert np.array_equal(vc.cpu().numpy().view(np.uint32), ovc)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("random_level", [True, False])
def test_hec_v3_map_bit_exact(partitioner, name, random_level):
    g = CASES[name]
    rp, col, w = dev(g)
    seed = 0x1234ABCD
    vc, nc, _ = partitioner.coarsen_map(rp, col, w, L.COARSEN_HEC_V3, random_level, seed)
    ovc, onc = O.hec_v3_map(g.row_ptr, g.col, g.w, random_level, seed)
    assert nc == onc and np.array_equal(vc.cpu().numpy().view(np.uint32), ovc)


@pytest.mark.parametrize("name", sorted(CASES))
def test_gosh_v2_map_bit_exact(partitioner, name):
    g = CASES[name]
    rp, col, w = dev(g)
    seed = 0x77AB
    vc, nc, _ = partitioner.coarsen_map(rp, col, w, L.COARSEN_GOSH_V2, False, seed)
    ovc, onc = O.gosh_v2_map(g.row_ptr, g.col, g.w, seed)
    assert nc == onc and np.array_equal(vc.cpu().numpy().view(np.uint32), ovc)


def test_coarsen_map_rejects_hec(partitioner):
    rp, col, _ = dev(CASES["grid"])
    with pytest.raises(L.SgparError):
        partitioner.coarsen_map(rp, col, None, L.COARSEN_HEC, False, 1)


def cut_of(g, labels):
    r = np.repeat(np.arange(g.n), np.diff(g.row_ptr).astype(np.int64))
    return int((labels[r] != labels[g.col]).sum()) // 2


@pytest.mark.parametrize("coarsener", [L.COARSEN_MATCH, L.COARSEN_MIS2, L.COARSEN_GOSH, L.COARSEN_HEC_V3,
                                       L.COARSEN_GOSH_V2,
                                       L.COARSEN_MATCH | L.COARSEN_RATIO_STOP, L.COARSEN_NONE])
@pytest.mark.parametrize("name", ["holes", "rmat14", "er_small"])
def test_partition_with_coarsener(partitioner, coarsener, name):
    if coarsener == L.COARSEN_NONE and name != "er_small":
        pytest.skip("the finest-level-only iteration converges slowly on these; covered on er_small")
    g = CASES[name] if name != "er_small" else G.erdos_renyi(3000, 6.0, seed=9)
    o = O.partition_graph(g.row_ptr, g.col, None, rng_state=21, coarsener=coarsener)
    r = partitioner.partition(g, rng_state=21, coarsener=coarsener)
    assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
    assert r.edgecut == cut_of(g, r.part)
    assert abs(r.edgecut - o["edgecut"]) <= 0.05 * o["edgecut"] + 4
    if coarsener != L.COARSEN_NONE:
        assert abs(r.lam - o["lambda"]) <= 1e-6 * abs(o["lambda"]) + 1e-12


def test_config_coarsening_alg_bits():
    """sgp_partition_graph: coarsening_alg & 1 -> matching with the 0.9
    ratio stop, & 16 -> no coarsening (sgpar.h:2457-2475)."""
    g = G.erdos_renyi(3000, 6.0, seed=9)
    for alg, coarsener in ((5, L.COARSEN_MATCH | L.COARSEN_RATIO_STOP), (16, L.COARSEN_NONE), (4, 0)):
        cfg = api.Config(coarsening_alg=alg, num_iter=1)
        part, cut = api.partition_graph(g, cfg, 0, api.PCG32(state=13, inc=1))
        o = O.partition_graph(g.row_ptr, g.col, None, rng_state=13, coarsener=coarsener)
        assert cut == cut_of(g, part)
        assert abs(cut - o["edgecut"]) <= 0.05 * o["edgecut"] + 4


def test_batch_and_4way_take_the_coarsener(partitioner):
    gs = [CASES["holes"], CASES["er"]]
    many = partitioner.partition_batch(gs, workers=2, rng_state=8, coarsener=L.COARSEN_GOSH)
    for g, r in zip(gs, many):
        s = partitioner.partition(g, rng_state=8, coarsener=L.COARSEN_GOSH, cluster_max_log2=23, cluster_blocks=2)
        assert np.array_equal(r.part, s.part) and r.level_n == s.level_n
    part4, cut2, cut4, _ = partitioner.partition_4way(CASES["holes"], rng_state=8, coarsener=L.COARSEN_MATCH)
    assert cut4 == cut_of(CASES["holes"], part4) and part4.max() <= 3
