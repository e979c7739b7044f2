"""The partitioning configurations at their full sizes, checked through
properties that hold at any size (the oracle takes minutes to hours there):

* R-MAT scale 22 (2.39M vertices after LCC, 64M edges): FP64 and mixed
  precision, balanced parts, the reported cut equal to the cut recomputed from
  the partition, the mixed cut within 1% of the FP64 cut and its Fiedler
  value within 1e-6 relative of the FP64 one;
* weighted Chung-Lu, 8,388,608 vertices, ~1e8 edges, weights in [1, 100]:
  the heavy-edge mapping passes the HEC validity check, and the coarse graph
  built from it with 64-bit weights conserves the fine weights exactly (total
  and two position-weighted checksums over (coarse u, coarse v)), rows
  strictly sorted with no self loops, the mapping onto [0, nc);
* 3D random geometric graph, 2^24 points, mean degree ~12: the 4-way driver
  (balanced quarters, cut2 <= cut4, both recomputed);
* the batch of 2,048 graphs of 1e3..2.5e5 vertices (grids with holes and
  Erdos-Renyi): every result balanced and its cut recomputed, a sample equal
  to single calls bit for bit.

The cut and checksum arithmetic runs on the GPU with torch (int64)."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import graphs as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).astype(np.int64)).cuda()


def rows_of(row_ptr):
    deg = dev(np.diff(row_ptr.astype(np.int64)))
    return torch.repeat_interleave(torch.arange(deg.numel(), device="cuda"), deg)


def cut_dev(g, labels):
    """Undirected edges whose endpoints carry different labels."""
    lab = dev(labels)
    r = rows_of(g.row_ptr)
    return int((lab[r] != lab[dev(g.col)]).sum().item()) // 2


def check_bisection(g, r):
    part = np.asarray(r.part)
    assert int((part == 0).sum()) in (g.n // 2, (g.n + 1) // 2)
    assert r.edgecut == cut_dev(g, part)
    assert r.lam > 0 and not r.iter_max_reached
    assert all(a > b for a, b in zip(r.level_n, r.level_n[1:]))


def test_rmat22_fp64_and_mixed(partitioner):
    g = G.rmat(22, seed=1)
    r = partitioner.partition(g, rng_state=1)
    check_bisection(g, r)
    assert r.residual < 1e-3
    m = partitioner.partition(g, rng_state=1, mixed=True)
    check_bisection(g, m)
    assert m.level_n == r.level_n
    assert abs(m.edgecut - r.edgecut) <= 0.01 * r.edgecut
    assert abs(m.lam - r.lam) <= 1e-6 * r.lam


def test_chunglu23_weighted_coarse_weights_conserved(partitioner):
    from oracle import bindings as O
    g = G.chung_lu(1 << 23, wmax=100, seed=1)
    assert 0.8e8 < g.m_directed // 2 < 1.2e8
    i32 = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()
    rp, col, w32 = i32(g.row_ptr), i32(g.col), i32(g.w)
    hn, vc32, nc, _ = partitioner.hec(rp, col, w32, random_level=False, seed=5)
    assert O.hec_check(hn.cpu().numpy().view(np.uint32), vc32.cpu().numpy().view(np.uint32), nc) == 0
    # 64-bit coarse weights: the total weight exceeds 2^32
    crp, ccol, cw = partitioner.build_coarse(rp, col, w32, vc32, nc, out_wbytes=8)
    vc = vc32.to(torch.int64)
    assert int(vc.max().item()) < nc and bool((torch.bincount(vc, minlength=nc) > 0).all())
    # fine entries mapped to coarse pairs, self loops of aggregates dropped
    cu = vc[rows_of(g.row_ptr)]
    cv = vc[dev(g.col)]
    w = dev(g.w)
    keep = cu != cv
    cu, cv, w = cu[keep], cv[keep], w[keep]
    crp = crp.to(torch.int64)
    ccol = ccol.to(torch.int64)
    crow = torch.repeat_interleave(torch.arange(nc, device="cuda"), crp[1:] - crp[:-1])
    assert bool((crow != ccol).all())
    same_row = crow[1:] == crow[:-1]
    assert bool((ccol[1:][same_row] > ccol[:-1][same_row]).all())
    assert int(cw.min().item()) >= 1 and int(cw.sum().item()) > 0xFFFFFFFF
    assert int(cw.sum().item()) == int(w.sum().item())
    for mul in (1000003, 7919):
        f = lambda a, b: (a * mul + b) & 0xFFFF
        assert int((cw * f(crow, ccol)).sum().item()) == int((w * f(cu, cv)).sum().item())
    del cu, cv, w, crow, ccol, cw, vc, crp, rp, col, w32, hn, vc32
    r = partitioner.partition(g, rng_state=3)
    check_bisection(g, r)


def test_rgg24_4way(partitioner):
    g = G.rgg3d(1 << 24, seed=1)
    part4, cut2, cut4, _ = partitioner.partition_4way(g, rng_state=5)
    part4 = np.asarray(part4)
    sizes = np.bincount(part4, minlength=4)
    assert sizes.sum() == g.n and sizes.max() - sizes.min() <= 2
    assert cut4 == cut_dev(g, part4) and cut2 == cut_dev(g, part4 >> 1) and cut2 <= cut4


def test_batch2048(partitioner):
    rng = np.random.default_rng(2048)
    sizes = np.exp(rng.uniform(np.log(1000), np.log(250000), 2048)).astype(int)
    gs = []
    for i, s in enumerate(sizes):
        if i % 2 == 0:
            nx = int(np.sqrt(s))
            gs.append(G.grid2d_holes(nx, max(2, int(s) // nx), seed=i + 1))
        else:
            gs.append(G.erdos_renyi(int(s), 8.0, seed=i + 1))
    rs = partitioner.partition_batch(gs, workers=8, rng_state=11)
    assert len(rs) == len(gs)
    for g, r in zip(gs, rs):
        part = np.asarray(r.part)
        assert int((part == 0).sum()) in (g.n // 2, (g.n + 1) // 2)
        rows = np.repeat(np.arange(g.n), np.diff(g.row_ptr).astype(np.int64))
        assert r.edgecut == int((part[rows] != part[g.col]).sum()) // 2
    for k in (0, 1, 777, 1500, 2047):
        s = partitioner.partition(gs[k], rng_state=11, cluster_max_log2=23, cluster_blocks=2)
        assert np.array_equal(np.asarray(rs[k].part), np.asarray(s.part)) and rs[k].edgecut == s.edgecut
        assert rs[k].level_iters == s.level_iters
