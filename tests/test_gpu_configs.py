"""The parity configurations of the partitioning path beyond R-MAT, at sizes
the oracle finishes in seconds: the 256x256 grid with coarsening cutoff 32,
the reference driver's 4-way mode on a 3D random geometric graph, a batch of
small grids-with-holes and Erdos-Renyi graphs, and weighted Chung-Lu inputs
(32-bit and 64-bit coarse weights).

Integer results (hierarchy sizes, rng advance, cuts recomputed from the
partition) are compared exactly; FP64 results within the tolerances stated
in each test.
"""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O

pytestmark = pytest.mark.gpu


def cut_of(g, labels):
    """Undirected edges whose endpoints carry different labels."""
    rows = np.repeat(np.arange(g.n), np.diff(g.row_ptr).astype(np.int64))
    return int((labels[rows] != labels[g.col]).sum()) // 2


def test_grid256_cutoff32(partitioner):
    g = G.grid2d(256, 256)
    o = O.partition_graph(g.row_ptr, g.col, None, cutoff=32, tol=1e-10, rng_state=7)
    r = partitioner.partition(g, cutoff=32, tol=1e-10, rng_state=7)
    assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
    assert r.edgecut == cut_of(g, r.part)
    assert int(r.part.sum()) == g.n // 2
    # FP64 power iteration: same stopping rule, summation order differs
    assert abs(r.lam - o["lambda"]) <= 1e-6 * o["lambda"]
    assert abs(r.edgecut - o["edgecut"]) <= 0.05 * o["edgecut"] + 4
    # the finest iterate approximates the Fiedler pair of the grid:
    # lambda_2 = 2 - 2 cos(pi / 256); the reference's stopping rule ends
    # within 5% of it (3.2% for this seed)
    lam2 = 2 - 2 * np.cos(np.pi / 256)
    assert 0 <= (r.lam - lam2) / lam2 < 0.05


def oracle_4way(g, rng_state, cutoff=50):
    """sgpar.cpp:62-89 on the oracle: bisection, induced subgraphs, one
    bisection of each with the rng carried on."""
    o = O.partition_graph(g.row_ptr, g.col, None, cutoff=cutoff, tol=1e-10, rng_state=rng_state)
    (rp1, c1), (rp2, c2) = O.use_partition(g.row_ptr, g.col, o["part"])
    st = o["rng_state"]
    cuts = [o["edgecut"]]
    for rp, c in ((rp1, c1), (rp2, c2)):
        s = O.partition_graph(rp, c, None, cutoff=cutoff, tol=1e-10, rng_state=st)
        st = s["rng_state"]
        cuts.append(s["edgecut"])
    return cuts, st


def test_rgg_4way_matches_driver(partitioner):
    g = G.rgg3d(20000, seed=3)
    part4, cut2, cut4, st = partitioner.partition_4way(g, rng_state=11)
    # the bisection is the plain partition with the same seed
    r = partitioner.partition(g, rng_state=11)
    assert np.array_equal(part4 >> 1, r.part) and cut2 == r.edgecut
    # labels 0..3, each half split in halves, cut4 counts every cut edge once
    sizes = np.bincount(part4, minlength=4)
    assert part4.max() <= 3 and sizes.sum() == g.n
    n0 = int((r.part == 0).sum())
    assert sorted([sizes[0], sizes[1]]) == sorted([n0 // 2, n0 - n0 // 2])
    assert cut4 == cut_of(g, part4)
    # against the oracle driver: FP64 differences may move a few vertices
    ocuts, _ = oracle_4way(g, 11)
    assert abs(cut2 - ocuts[0]) <= 0.05 * ocuts[0] + 4
    assert abs(cut4 - sum(ocuts)) <= 0.05 * sum(ocuts) + 8


def test_4way_device_resident(partitioner):
    torch = pytest.importorskip("torch")
    g = G.grid2d_holes(120, 90, seed=2)
    dev = {"row_ptr": torch.from_numpy(g.row_ptr.view(np.int32)).cuda(),
           "col": torch.from_numpy(g.col.view(np.int32)).cuda()}
    out = torch.zeros(g.n, dtype=torch.int32, device="cuda")
    _, cut2, cut4, _ = partitioner.partition_4way(dev, rng_state=5, part_out=out)
    host, h2, h4, _ = partitioner.partition_4way(g, rng_state=5)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), host) and (cut2, cut4) == (h2, h4)


def batch_graphs(count, seed=17, lo=1000, hi=12000):
    """Vertex counts log-uniform in [lo, hi]; even indices grids with 10% of
    the vertices removed, odd ones Erdos-Renyi of mean degree 8 (LCC)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(int)
    out = []
    for i, s in enumerate(sizes):
        if i % 2 == 0:
            nx = int(np.sqrt(s))
            out.append(G.grid2d_holes(nx, max(2, int(s) // nx), seed=i + 1))
        else:
            out.append(G.erdos_renyi(int(s), 8.0, seed=i + 1))
    return out


# a batch runs levels of up to 2^23 cost units on the cluster kernel in
# clusters of 2 blocks (single calls: 2^17, 8 blocks); with the same
# cluster_max_log2 and cluster_blocks a single call gives equal bits
BATCH_CLUSTER = 23
BATCH_BLOCKS = 2


def test_batch_equals_single_calls(partitioner):
    gs = batch_graphs(12)
    many = partitioner.partition_batch(gs, workers=4, rng_state=9)
    one = partitioner.partition_batch(gs, workers=1, rng_state=9)
    for g, a, b in zip(gs, many, one):
        s = partitioner.partition(g, rng_state=9, cluster_max_log2=BATCH_CLUSTER, cluster_blocks=BATCH_BLOCKS)
        for r in (a, b):
            assert np.array_equal(r.part, s.part)
            assert r.edgecut == s.edgecut == cut_of(g, r.part)
            assert r.level_iters == s.level_iters and r.rng_state == s.rng_state


def same_result(a, b):
    assert np.array_equal(a.part, b.part) and a.edgecut == b.edgecut
    assert a.level_n == b.level_n and a.level_iters == b.level_iters and a.rng_state == b.rng_state
    assert a.lam == b.lam and a.residual == b.residual


def test_batch_of_small_hierarchies(partitioner):
    """Graphs whose every level, level 0 included, is a small level: the
    whole eigensolve of each is the batch's one chained launch (one block per
    hierarchy), and the result equals a single call's bit for bit."""
    gs = batch_graphs(40, seed=5, lo=40, hi=1500)
    rs = partitioner.partition_batch(gs, workers=3, rng_state=2)
    for g, r in zip(gs, rs):
        same_result(r, partitioner.partition(g, rng_state=2, cluster_max_log2=BATCH_CLUSTER,
                                             cluster_blocks=BATCH_BLOCKS))
        assert r.edgecut == cut_of(g, r.part)
    for g, r in list(zip(gs, rs))[:6]:
        o = O.partition_graph(g.row_ptr, g.col, None, cutoff=50, tol=1e-10, rng_state=2)
        assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
        assert abs(r.lam - o["lambda"]) <= 1e-6 * abs(o["lambda"])


@pytest.mark.parametrize("mixed", [False, True])
def test_batch_weighted_and_mixed_equal_single_calls(partitioner, mixed):
    """64-bit coarse weights (total weight above 2^32) and the mixed-precision
    path through the batch: each graph as a single call."""
    gs = [G.chung_lu(n, wmax=1 << 22, seed=s) for n, s in ((3000, 1), (9000, 2), (600, 3))]
    gs += batch_graphs(5, seed=41, lo=2000, hi=20000)
    rs = partitioner.partition_batch(gs, workers=2, rng_state=8, mixed=mixed)
    for g, r in zip(gs, rs):
        same_result(r, partitioner.partition(g, rng_state=8, mixed=mixed, cluster_max_log2=BATCH_CLUSTER,
                                             cluster_blocks=BATCH_BLOCKS))


def test_batch_default_and_single_default_agree(partitioner):
    """Default settings: the batch's mid-size levels run on the cluster kernel
    and a single call's larger ones on the whole GPU; the hierarchy and rng
    are the same, the Fiedler values agree to rounding and the cuts to 1%."""
    gs = batch_graphs(6, seed=29, lo=5000, hi=40000)
    rs = partitioner.partition_batch(gs, workers=3, rng_state=12)
    for g, r in zip(gs, rs):
        s = partitioner.partition(g, rng_state=12)
        assert r.level_n == s.level_n and r.rng_state == s.rng_state
        assert abs(r.lam - s.lam) <= 1e-8 * abs(s.lam)
        assert abs(r.edgecut - s.edgecut) <= 0.01 * s.edgecut and r.edgecut == cut_of(g, r.part)


def test_batch_matches_oracle(partitioner):
    gs = batch_graphs(6, seed=23)
    rs = partitioner.partition_batch(gs, workers=3, rng_state=4)
    for g, r in zip(gs, rs):
        o = O.partition_graph(g.row_ptr, g.col, None, cutoff=50, tol=1e-10, rng_state=4)
        assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
        assert abs(r.edgecut - o["edgecut"]) <= 0.05 * o["edgecut"] + 4


def test_batch_reports_the_failing_graph(partitioner):
    from ipdps_2021_graph_coarsening_b200 import _lib as L
    gs = batch_graphs(3)
    bad = G.CSR(gs[1].row_ptr.copy(), gs[1].col.copy())
    bad.col[0] = bad.n + 5   # destination out of range
    with pytest.raises(L.SgparError) as e:
        partitioner.partition_batch([gs[0], bad, gs[2]], workers=2)
    assert "graph 1" in str(e.value)


@pytest.mark.parametrize("wmax", [100, 1 << 22])
def test_chunglu_weighted(partitioner, wmax):
    """Weighted input; wmax 2^22 makes the total weight exceed 2^32, so the
    coarse weights are 64-bit."""
    g = G.chung_lu(20000, wmax=wmax, seed=5)
    assert g.w is not None
    total = int(g.w.astype(np.uint64).sum())
    assert (total > 0xFFFFFFFF) == (wmax > 1000)
    o = O.partition_graph(g.row_ptr, g.col, g.w, cutoff=50, tol=1e-10, rng_state=3)
    r = partitioner.partition(g, cutoff=50, tol=1e-10, rng_state=3)
    assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
    assert r.edgecut == cut_of(g, r.part)
    assert abs(r.lam - o["lambda"]) <= 1e-6 * abs(o["lambda"])
    assert abs(r.edgecut - o["edgecut"]) <= 0.05 * o["edgecut"] + 4


def test_sharded_batch_on_one_rank(partitioner):
    """The multi-rank batch driver on a single rank runs the whole batch
    through the batched entry point, in the graphs' order."""
    from ipdps_2021_graph_coarsening_b200 import shard
    gs = batch_graphs(5, seed=31)
    out = shard.partition_sharded(gs, lambda l: partitioner.partition_batch(l, workers=2, rng_state=6), 0, 1)
    for g, r in zip(gs, out):
        s = partitioner.partition(g, rng_state=6, cluster_max_log2=BATCH_CLUSTER, cluster_blocks=BATCH_BLOCKS)
        assert np.array_equal(r.part, s.part) and r.edgecut == s.edgecut


def test_metrics_record_of_a_partition(partitioner, tmp_path):
    """A real partition written in the reference's metrics layout: phase
    times add up and the levels match the result."""
    import json
    from ipdps_2021_graph_coarsening_b200.api import write_metrics
    g = G.rmat(13, seed=3)
    r = partitioner.partition(g, rng_state=2)
    part4, _, cut4, _ = partitioner.partition_4way(g, rng_state=2)
    path = str(tmp_path / "m.json")
    write_metrics(path, r, edge_cut_4way=cut4)
    (d,) = json.load(open(path))
    assert d["edge-cut"] == r.edgecut and d["edge-cut-four-way"] == cut4
    assert d["number-coarse-levels"] == r.levels == len(d["coarse-levels"])
    assert [x["number-vertices"] for x in d["coarse-levels"]] == r.level_n[::-1]
    assert [x["refine-iterations"] for x in d["coarse-levels"]] == r.level_iters[::-1]
    assert 0 < d["coarsen-map-duration-seconds"] + d["coarsen-build-duration-seconds"] <= d["coarsen-duration-seconds"]
    assert d["total-duration-seconds"] > d["refine-duration-seconds"] > 0


@pytest.mark.parametrize("name", ["grid64", "holes", "rmat12"])
def test_normalized_laplacian_variant(partitioner, name):
    """refine_alg 1 (eigensolve_kokkos.h:103-206): the lazy random walk with
    a D-orthogonalised start and no deflation in the loop.  On grids it finds
    the normalized Fiedler pair like the oracle; on R-MAT levels the constant
    vector grows back from rounding and both collapse onto it (lambda ~ 0),
    as the reference does."""
    g = {"grid64": lambda: G.grid2d(64, 64), "holes": lambda: G.grid2d_holes(60, 60, 0.1, 4),
         "rmat12": lambda: G.rmat(12, seed=3)}[name]()
    o = O.partition_graph(g.row_ptr, g.col, None, rng_state=77, refine_alg=1)
    r = partitioner.partition(g, rng_state=77, refine_alg=1)
    assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
    assert r.edgecut == cut_of(g, r.part)
    assert int((r.part == 0).sum()) in (g.n // 2, (g.n + 1) // 2)
    if name == "rmat12":
        assert abs(r.lam) < 1e-4 and abs(o["lambda"]) < 1e-4
    else:
        # same hierarchy and iteration counts as the oracle: FP64 agrees to
        # rounding, mixed precision within the 1e-6 bound of the other tests
        assert r.level_iters == o["level_iters"]
        assert abs(r.lam - o["lambda"]) <= 1e-8 * o["lambda"]
        assert abs(r.edgecut - o["edgecut"]) <= 0.05 * o["edgecut"] + 4
        rm = partitioner.partition(g, rng_state=77, refine_alg=1, mixed=True)
        assert abs(rm.lam - o["lambda"]) <= 1e-6 * o["lambda"]
        # and it differs from the combinatorial variant's eigenvalue
        c = partitioner.partition(g, rng_state=77)
        assert abs(c.lam - r.lam) > 0.5 * r.lam


def test_refine_alg_out_of_range_is_rejected(partitioner):
    from ipdps_2021_graph_coarsening_b200 import _lib as L
    with pytest.raises(L.SgparError):
        partitioner.partition(G.grid2d(20, 20), refine_alg=2)


def test_cluster_blocks_option(partitioner):
    """Clusters of 2 and 8 blocks for the mid-size levels (the 300 x 300
    grid's level of 3243 vertices runs there) give the same hierarchy and
    agree to rounding; other block counts are rejected."""
    g = G.grid2d(300, 300)
    a = partitioner.partition(g, rng_state=3, cluster_blocks=2)
    b = partitioner.partition(g, rng_state=3, cluster_blocks=8)
    c = partitioner.partition(g, rng_state=3)
    assert a.level_n == b.level_n == c.level_n and a.rng_state == b.rng_state
    assert b.lam == c.lam and b.edgecut == c.edgecut   # 8 is the single-call default
    assert abs(a.lam - b.lam) <= 1e-8 * abs(b.lam)
    assert abs(a.edgecut - b.edgecut) <= 0.01 * b.edgecut
    with pytest.raises(L.SgparError) as ei:
        partitioner.partition(g, rng_state=3, cluster_blocks=3)
    assert ei.value.code == L.ERR_INVALID and "cluster_blocks" in L.last_error()
