"""The edge-case graphs (a single vertex, a single edge, two components, a long
path, a star, a complete graph, an odd cycle) through the alternative
coarseners, the local search and FM: the device path against the oracle
(hierarchies, rng advance and FM moves exactly; local search bit-exact against
the reference's own build where it is present)."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import api
from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O
from tests.test_gpu_edge_cases import CASES, cut_of

pytestmark = pytest.mark.gpu

COARSENERS = [L.COARSEN_MATCH, L.COARSEN_MIS2, L.COARSEN_GOSH, L.COARSEN_HEC_V3, L.COARSEN_GOSH_V2]


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("coarsener", COARSENERS)
def test_coarseners_on_edge_cases(partitioner, name, coarsener):
    g = CASES[name]()
    o = O.partition_graph(g.row_ptr, g.col, None, rng_state=13, coarsener=coarsener)
    r = partitioner.partition(g, rng_state=13, coarsener=coarsener)
    assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
    part = np.asarray(r.part)
    assert int((part == 0).sum()) in (g.n // 2, (g.n + 1) // 2)
    assert r.edgecut == cut_of(g, part)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fm_on_edge_cases(partitioner, name):
    g = CASES[name]()
    base = partitioner.partition(g, rng_state=13)
    r = partitioner.partition(g, rng_state=13, fm_passes=8)
    op, oc, opasses, omoves = O.fm_refine(g.row_ptr, g.col, None, np.asarray(base.part), 8)
    assert np.array_equal(np.asarray(r.part), op) and r.edgecut == oc == cut_of(g, np.asarray(r.part))
    assert r.edgecut <= base.edgecut and (r.fm_passes, r.fm_moves) == (opasses, omoves)


@pytest.mark.parametrize("name", sorted(CASES))
def test_local_search_on_edge_cases(name):
    g = CASES[name]()
    ev = O.partition_graph(g.row_ptr, g.col, None, rng_state=13)["evec"]
    part, cut = api.compute_partition(ev, g, 2, 0, local_search_alg=1)
    op, oc, _ = O.compute_partition_ls(g.row_ptr, g.col, ev)
    assert np.array_equal(part, op) and cut == oc == cut_of(g, part)
    if O.ref_available("serial"):
        rp, rc = O.ref_compute_partition_ls(g.row_ptr, g.col, ev)
        assert np.array_equal(part, rp) and cut == rc


@pytest.mark.parametrize("name", ["grid", "rmat13", "chunglu_w"])
def test_hierarchy_levels_and_vertex_weights(partitioner, name):
    """The lower boundary (sgp_generate_coarse_graphs, coarsen_kokkos.h:1165):
    the device hierarchy equals the oracle's level sizes, each level's
    vertex weights are the previous level's summed over its aggregates
    (coarsen_kokkos.h:1098; level 0 has unit weights) and add up to the input's
    vertex count, and every coarse level is the oracle's build of the level
    above under the device's own mapping."""
    g = {"grid": lambda: G.grid2d(70, 50), "rmat13": lambda: G.rmat(13, seed=2),
         "chunglu_w": lambda: G.chung_lu(30000, wmax=50, seed=3)}[name]()
    rng = api.PCG32(state=99, inc=1)
    h = partitioner.generate_coarse_graphs(g, cutoff=50, rng=rng)
    try:
        o = O.partition_graph(g.row_ptr, g.col, g.w, cutoff=50, rng_state=99)
        assert [h.level(l)["n"] for l in range(len(h))] == o["level_n"]
        assert h.level(0)["vtx_w"] is None
        vw = np.ones(g.n, np.int64)
        for l in range(len(h) - 1):
            lv, nx = h.level(l), h.level(l + 1)
            vc = lv["vcmap"].cpu().numpy().view(np.uint32)
            want = np.bincount(vc, weights=vw, minlength=nx["n"]).astype(np.int64)
            got = nx["vtx_w"].cpu().numpy().view(np.uint32).astype(np.int64)
            assert np.array_equal(got, want)
            assert int(got.sum()) == g.n
            rp, col = lv["row_ptr"].cpu().numpy().view(np.uint32), lv["col"].cpu().numpy().view(np.uint32)
            w = None if lv["w"] is None else lv["w"].cpu().numpy().view(np.uint32 if lv["wbytes"] == 4 else np.uint64)
            crp, ccol, cw = O.build_coarse(rp, col, w, vc, nx["n"])
            assert np.array_equal(nx["row_ptr"].cpu().numpy().view(np.uint32), crp)
            assert np.array_equal(nx["col"].cpu().numpy().view(np.uint32), ccol)
            nw = nx["w"].cpu().numpy().view(np.uint32 if nx["wbytes"] == 4 else np.uint64)
            assert np.array_equal(nw.astype(np.uint64), cw)
            vw = got
    finally:
        h.free()
