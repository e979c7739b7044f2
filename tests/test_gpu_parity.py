"""Parity of the sm_100a path with the CPU oracle, through the C ABI.

Integer work (HEC mapping, coarse build, split, cut) must be bit-exact.
FP64 power iteration follows the reference's recurrence with a different
summation order, so eigen results are compared with stated tolerances:
  * Rayleigh quotient relative error <= 1e-6 against the oracle run from the
    same start vector (and <= 1e-9 when both ran the same iteration count);
  * the returned unit vectors agree to |1 - <x_gpu, x_orc>| <= 1e-8 when the
    iteration counts agree.
"""
import numpy as np
import pytest

from oracle import bindings as O
from ipdps_2021_graph_coarsening_b200 import graphs as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev_u32(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def dev_u64(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).cuda()


def host_u32(t):
    return t.cpu().numpy().view(np.uint32)


def host_u64(t):
    return t.cpu().numpy().view(np.uint64)


def star_plus_ring(n_leaves=9000, ring=3000):
    """A hub joined to n_leaves leaves plus a ring: coarse rows above the
    shared-memory tier appear after one HEC level."""
    n = 1 + n_leaves + ring
    edges = [(0, i) for i in range(1, n_leaves + 1)]
    r0 = n_leaves + 1
    edges += [(r0 + i, r0 + (i + 1) % ring) for i in range(ring)]
    edges += [(i, r0 + (i * 7) % ring) for i in range(1, n_leaves + 1)]
    adj = [[] for _ in range(n)]
    for a, b in edges:
        adj[a].append(b)
        adj[b].append(a)
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum([len(set(x)) for x in adj])
    col = np.concatenate([np.array(sorted(set(x)), np.uint32) for x in adj])
    return G.CSR(rp, col)


GRAPHS = {
    "grid64": lambda: G.grid2d(64, 64),
    "grid_odd": lambda: G.grid2d(33, 47),
    "rmat12": lambda: G.rmat(12, seed=3),
    "er3000": lambda: G.erdos_renyi(3000, 8.0, seed=2),
    "holes": lambda: G.grid2d_holes(60, 60, 0.1, 4),
    "star": star_plus_ring,
}


@pytest.fixture(scope="module", params=sorted(GRAPHS))
def graph(request):
    return GRAPHS[request.param]()


# ------------------------------------------------------------------ HEC --
@pytest.mark.parametrize("random_level", [True, False])
def test_hec_bit_exact(partitioner, graph, random_level):
    seed = 0x1234_5678_9ABC_DEF0 + int(random_level)
    hn_o = O.hec_heavy(graph.row_ptr, graph.col, None, random_level, seed)
    vc_o, nc_o, rounds_o = O.hec_map(hn_o, seed)
    hn, vc, nc, rounds = partitioner.hec(dev_u32(graph.row_ptr), dev_u32(graph.col), None, random_level, seed)
    assert np.array_equal(host_u32(hn), hn_o)
    assert nc == nc_o
    assert np.array_equal(host_u32(vc), vc_o)
    assert rounds == rounds_o
    assert O.hec_check(hn_o, host_u32(vc), nc) == 0


def test_hec_weighted_levels_bit_exact(partitioner, graph):
    # a weighted graph: the oracle's first coarse level
    hn = O.hec_heavy(graph.row_ptr, graph.col, None, True, 7)
    vc, nc, _ = O.hec_map(hn, 7)
    crp, ccol, cw = O.build_coarse(graph.row_ptr, graph.col, None, vc, nc)
    for wdt in ("u32", "u64"):
        wdev = dev_u32(cw) if wdt == "u32" else dev_u64(cw)
        seed = 99
        hn_o = O.hec_heavy(crp, ccol, cw, False, seed)
        vc_o, nc_o, _ = O.hec_map(hn_o, seed)
        hn_g, vc_g, nc_g, _ = partitioner.hec(dev_u32(crp), dev_u32(ccol), wdev, False, seed)
        assert np.array_equal(host_u32(hn_g), hn_o)
        assert nc_g == nc_o and np.array_equal(host_u32(vc_g), vc_o)


# ---------------------------------------------------------------- build --
@pytest.mark.parametrize("out_wbytes", [4, 8])
def test_build_bit_exact(partitioner, graph, out_wbytes):
    hn = O.hec_heavy(graph.row_ptr, graph.col, None, True, 21)
    vc, nc, _ = O.hec_map(hn, 21)
    rp_o, col_o, w_o = O.build_coarse(graph.row_ptr, graph.col, None, vc, nc)
    crp, ccol, cw = partitioner.build_coarse(dev_u32(graph.row_ptr), dev_u32(graph.col), None, dev_u32(vc), nc,
                                             out_wbytes)
    assert np.array_equal(host_u32(crp), rp_o)
    assert np.array_equal(host_u32(ccol), col_o)
    w = host_u32(cw) if out_wbytes == 4 else host_u64(cw)
    assert np.array_equal(w.astype(np.uint64), w_o)
    # second level: weighted input
    hn2 = O.hec_heavy(rp_o, col_o, w_o, False, 22)
    vc2, nc2, _ = O.hec_map(hn2, 22)
    rp2, col2, w2 = O.build_coarse(rp_o, col_o, w_o, vc2, nc2)
    win = dev_u32(w_o) if out_wbytes == 4 else dev_u64(w_o)
    g_rp, g_col, g_w = partitioner.build_coarse(dev_u32(rp_o), dev_u32(col_o), win, dev_u32(vc2), nc2, out_wbytes)
    assert np.array_equal(host_u32(g_rp), rp2)
    assert np.array_equal(host_u32(g_col), col2)
    gw = host_u32(g_w) if out_wbytes == 4 else host_u64(g_w)
    assert np.array_equal(gw.astype(np.uint64), w2)


@pytest.mark.parametrize("n_leaves,ring", [(12000, 4000), (67500, 22500), (90000, 30000)])
@pytest.mark.parametrize("out_wbytes", [4, 8])
def test_build_large_rows_dense_tier(partitioner, n_leaves, ring, out_wbytes):
    """Buckets above 4096 entries (the dense tier), with 8002 coarse vertices
    (several accumulator copies in one block's shared memory), 45002 (one
    copy and a bitmap with 32-bit weights; global memory with 64-bit ones)
    and 60002 (global memory), 32- and 64-bit coarse weights."""
    g = star_plus_ring(n_leaves, ring)
    # map everything in the first half to one aggregate: one huge bucket
    n = g.n
    vc = np.zeros(n, np.uint32)
    vc[n // 2:] = np.arange(1, n - n // 2 + 1, dtype=np.uint32)
    nc = int(vc.max()) + 1
    rp_o, col_o, w_o = O.build_coarse(g.row_ptr, g.col, None, vc, nc)
    crp, ccol, cw = partitioner.build_coarse(dev_u32(g.row_ptr), dev_u32(g.col), None, dev_u32(vc), nc, out_wbytes)
    assert int(np.diff(rp_o).max()) > 4096
    assert np.array_equal(host_u32(crp), rp_o)
    assert np.array_equal(host_u32(ccol), col_o)
    cwh = host_u32(cw).astype(np.uint64) if out_wbytes == 4 else host_u64(cw)
    assert np.array_equal(cwh, w_o)


@pytest.mark.parametrize("nc_tail", [20000, 70000])
@pytest.mark.parametrize("out_wbytes", [4, 8])
def test_build_giant_rows(partitioner, nc_tail, out_wbytes):
    """A bucket of more than 2^18 entries (split over many blocks) beside
    rows of the other tiers; the remaining vertices folded onto nc_tail
    coarse vertices (the shared-memory or the global dense tier)."""
    g = star_plus_ring(220000, 60000)
    n = g.n
    vc = np.zeros(n, np.uint32)
    vc[n // 2:] = 1 + (np.arange(n - n // 2, dtype=np.uint32) % nc_tail)
    nc = int(vc.max()) + 1
    rp_o, col_o, w_o = O.build_coarse(g.row_ptr, g.col, None, vc, nc)
    assert int(np.diff(rp_o).max()) > 0
    sizes = np.bincount(vc, weights=np.diff(g.row_ptr).astype(np.int64), minlength=nc)
    assert sizes.max() > (1 << 18)
    crp, ccol, cw = partitioner.build_coarse(dev_u32(g.row_ptr), dev_u32(g.col), None, dev_u32(vc), nc, out_wbytes)
    assert np.array_equal(host_u32(crp), rp_o)
    assert np.array_equal(host_u32(ccol), col_o)
    cwh = host_u32(cw).astype(np.uint64) if out_wbytes == 4 else host_u64(cw)
    assert np.array_equal(cwh, w_o)


# ---------------------------------------------------------------- split --
@pytest.mark.parametrize("ties", [False, True])
def test_split_bit_exact(partitioner, graph, ties):
    rng = np.random.default_rng(graph.n + int(ties))
    ev = rng.standard_normal(graph.n)
    if ties:
        ev = np.round(ev, 1)
        ev[::5] = 0.0
        ev[1::11] = -0.0
    p_o, c_o = O.compute_partition(graph.row_ptr, graph.col, ev)
    part, cut = partitioner.split(dev_u32(graph.row_ptr), dev_u32(graph.col), torch.from_numpy(ev).cuda())
    assert cut == c_o
    assert np.array_equal(host_u32(part), p_o)


# ------------------------------------------------------ power iteration --
@pytest.fixture(params=["auto", "stream", "row4", "rowp", "panel"])
def spmv_variant(request, monkeypatch):
    """Every SpMV variant of the power-iteration kernel (the default picks one
    per level by mean degree; the others are forced here)."""
    if request.param != "auto":
        monkeypatch.setenv("SGPB_PI_MODE", request.param)
    return request.param


@pytest.mark.parametrize("weighted", [False, True])
def test_power_iter_matches_oracle(partitioner, graph, weighted, spmv_variant):
    rp, col, w = graph.row_ptr, graph.col, None
    if weighted:
        hn = O.hec_heavy(rp, col, None, True, 5)
        vc, nc, _ = O.hec_map(hn, 5)
        rp, col, w = O.build_coarse(rp, col, None, vc, nc)
    n = rp.shape[0] - 1
    x0 = np.random.default_rng(n).random(n)
    cap = 4000
    u_o, it_o, lam_o = O.power_iter(rp, col, w, x0, 1e-10, cap)
    u_g, it_g, lam_g, res_g = partitioner.power_iter(dev_u32(rp), dev_u32(col), None if w is None else dev_u32(w),
                                                     torch.from_numpy(x0).cuda(), None, 1e-10, cap)
    u_g = u_g.cpu().numpy()
    assert abs(it_g - it_o) <= max(2, it_o // 50)
    assert abs(lam_g - lam_o) <= 1e-6 * abs(lam_o)
    if it_g == it_o:
        assert abs(lam_g - lam_o) <= 1e-9 * abs(lam_o) + 1e-15
        assert 1 - abs(float(np.dot(u_g, u_o))) <= 1e-8
    assert abs(np.linalg.norm(u_g) - 1) < 1e-9
    assert abs(u_g.sum()) < 1e-8 * np.sqrt(n)
    assert res_g >= 0


@pytest.mark.parametrize("weighted", [False, True])
def test_power_iter_column_panels(partitioner, weighted, monkeypatch):
    """Levels wider than one shared-memory panel (several panels per
    iteration in both precisions), against the oracle at a fixed iteration
    count."""
    monkeypatch.setenv("SGPB_PI_MODE", "panel")
    g = G.grid2d(250, 250)
    rp, col, w = g.row_ptr, g.col, None
    if weighted:
        hn = O.hec_heavy(rp, col, None, True, 8)
        vc, nc, _ = O.hec_map(hn, 8)
        rp, col, w = O.build_coarse(rp, col, None, vc, nc)
    n = rp.shape[0] - 1
    assert n > 12288   # more than one FP64 panel
    x0 = np.random.default_rng(n).random(n)
    cap = 300
    u_o, it_o, lam_o = O.power_iter(rp, col, w, x0, 1e-10, cap)
    u_g, it_g, lam_g, _ = partitioner.power_iter(dev_u32(rp), dev_u32(col), None if w is None else dev_u32(w),
                                                 torch.from_numpy(x0).cuda(), None, 1e-10, cap)
    assert it_g == it_o == cap
    assert abs(lam_g - lam_o) <= 1e-9 * abs(lam_o)
    assert 1 - abs(float(np.dot(u_g.cpu().numpy(), u_o))) <= 1e-9


def test_power_iter_panels_level_too_wide(partitioner, monkeypatch):
    """A level wider than the largest panel layout (409,600 vertices: 34 FP64
    panels of 12,288 entries, more than 31) keeps its rule variant when
    panels are asked for, and matches the oracle."""
    monkeypatch.setenv("SGPB_PI_MODE", "panel")
    g = G.grid2d(640, 640)
    assert g.n > 31 * 12288
    x0 = np.random.default_rng(6).random(g.n)
    cap = 40
    u_o, it_o, lam_o = O.power_iter(g.row_ptr, g.col, None, x0, 1e-10, cap)
    u_g, it_g, lam_g, _ = partitioner.power_iter(dev_u32(g.row_ptr), dev_u32(g.col), None,
                                                 torch.from_numpy(x0).cuda(), None, 1e-10, cap)
    assert it_g == it_o == cap
    assert abs(lam_g - lam_o) <= 1e-9 * abs(lam_o)
    assert 1 - abs(float(np.dot(u_g.cpu().numpy(), u_o))) <= 1e-9


def test_power_iter_panels_unsorted_rows(partitioner, monkeypatch):
    """Rows that are not ascending by destination cannot be cut into panel
    segments: the level runs on warp rows and still matches the oracle."""
    monkeypatch.setenv("SGPB_PI_MODE", "panel")
    g = G.grid2d(60, 60)
    rp, col = g.row_ptr, g.col.copy()
    for i in range(g.n):
        col[rp[i]:rp[i + 1]] = col[rp[i]:rp[i + 1]][::-1]
    x0 = np.random.default_rng(4).random(g.n)
    u_o, it_o, lam_o = O.power_iter(rp, col, None, x0, 1e-10, 200)
    u_g, it_g, lam_g, _ = partitioner.power_iter(dev_u32(rp), dev_u32(col), None, torch.from_numpy(x0).cuda(), None,
                                                 1e-10, 200)
    assert it_g == it_o
    assert abs(lam_g - lam_o) <= 1e-9 * abs(lam_o)


def test_partition_column_panels(partitioner, monkeypatch):
    """The whole path with every level on column panels, FP64 and mixed."""
    monkeypatch.setenv("SGPB_PI_MODE", "panel")
    g = G.rmat(13, seed=3)
    o = O.partition_graph(g.row_ptr, g.col, None, cutoff=50, tol=1e-10, rng_state=5)
    r = partitioner.partition(g, cutoff=50, tol=1e-10, rng_state=5)
    assert r.level_n == o["level_n"]
    assert r.edgecut == O.edge_cut(g.row_ptr, g.col, r.part)
    assert abs(r.edgecut - o["edgecut"]) <= 0.02 * o["edgecut"] + 2
    assert abs(r.lam - o["lambda"]) <= 1e-6 * abs(o["lambda"]) + 1e-12
    # mixed precision has no column-panel form: its levels take the warp-row kernel
    rm = partitioner.partition(g, cutoff=50, tol=1e-10, rng_state=5, mixed=True)
    assert abs(rm.lam - o["lambda"]) <= 1e-6 * abs(o["lambda"])


def rmat18_level1():
    g = G.rmat(18, seed=2)
    hn = O.hec_heavy(g.row_ptr, g.col, None, True, 5)
    vc, nc, _ = O.hec_map(hn, 5)
    return O.build_coarse(g.row_ptr, g.col, None, vc, nc)


@pytest.mark.parametrize("variant,wscale,wide", [("auto", 1, False), ("staged", 1, False), ("row4", 1, False),
                                                 ("stream", 1, False), ("auto", 300, False), ("staged", 300, False),
                                                 ("stream", 300, False), ("auto", 100000, False),
                                                 ("staged", 100000, False), ("auto", 7, True), ("staged", 7, True)])
@pytest.mark.parametrize("mixed", [False, True])
def test_power_iter_hub_first_copy(partitioner, monkeypatch, variant, wscale, wide, mixed):
    """A skewed level above 16384 vertices iterates on a hub-first
    relabelled copy whose leading entries are gathered through L1 and whose
    weights are stored in 8 bits (wscale 1: all weights <= 255), 16 bits
    (wscale 300), 32 bits (wscale 100000) or 64 bits (wide); its dense rows
    run on the register-pipelined warp rows by default ("auto") or on the
    staged ones ("staged": the matrix stream copied into shared memory by
    bulk copies).  The result (mapped back to the level's numbering) matches
    the run without the copy and the oracle, in both precisions."""
    rp, col, w = rmat18_level1()
    w = w * wscale
    assert int(w.max()) <= 0xFFFFFFFF and ((int(w.max()) <= 255) == (wscale == 1))
    n = rp.shape[0] - 1
    assert n > 16384
    assert rp[-1] > 64 * n   # dense: the warp-row variants
    if variant != "auto":
        monkeypatch.setenv("SGPB_PI_MODE", variant)
    x0 = torch.from_numpy(np.random.default_rng(n).random(n)).cuda()
    wd = dev_u64(w) if wide else dev_u32(w)
    args = (dev_u32(rp), dev_u32(col), wd, x0, None, 1e-10, 400, mixed)
    u_r, it_r, lam_r, res_r = partitioner.power_iter(*args)
    monkeypatch.setenv("SGPB_PI_RELABEL", "0")
    u_p, it_p, lam_p, _ = partitioner.power_iter(*args)
    assert abs(it_r - it_p) <= 2
    assert abs(lam_r - lam_p) <= 1e-9 * abs(lam_p)
    if it_r == it_p:
        assert 1 - abs(float(torch.dot(u_r, u_p))) <= 1e-9
    u_o, it_o, lam_o = O.power_iter(rp, col, w, x0.cpu().numpy(), 1e-10, 400)
    assert abs(it_r - it_o) <= max(2, it_o // 50)
    assert abs(lam_r - lam_o) <= 1e-6 * abs(lam_o)
    assert res_r >= 0


def test_power_iter_staged_unweighted(partitioner, monkeypatch):
    """Staged warp rows on an unweighted relabelled level (only destinations
    are copied), forced on the R-MAT 18 input graph, against the oracle."""
    g = G.rmat(18, seed=2)
    monkeypatch.setenv("SGPB_PI_MODE", "staged")
    x0 = np.random.default_rng(3).random(g.n)
    u_g, it_g, lam_g, _ = partitioner.power_iter(dev_u32(g.row_ptr), dev_u32(g.col), None,
                                                 torch.from_numpy(x0).cuda(), None, 1e-10, 300)
    u_o, it_o, lam_o = O.power_iter(g.row_ptr, g.col, None, x0, 1e-10, 300)
    assert abs(it_g - it_o) <= max(2, it_o // 50)
    assert abs(lam_g - lam_o) <= 1e-6 * abs(lam_o)
    if it_g == it_o:
        assert 1 - abs(float(np.dot(u_g.cpu().numpy(), u_o))) <= 1e-8


def test_partition_with_and_without_hub_first_copy(partitioner, monkeypatch):
    g = G.rmat(18, seed=2)
    a = partitioner.partition(g, rng_state=21)
    monkeypatch.setenv("SGPB_PI_RELABEL", "0")
    b = partitioner.partition(g, rng_state=21)
    assert a.level_n == b.level_n and a.rng_state == b.rng_state
    assert a.level_n[1] > 16384
    assert abs(a.edgecut - b.edgecut) <= 0.01 * b.edgecut
    assert abs(a.lam - b.lam) <= 1e-6 * abs(b.lam)


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("name", ["grid", "rmat10"])
def test_power_iter_small_level_kernel(partitioner, monkeypatch, weighted, name):
    """Levels that fit one block run on the shared-memory small-level kernel
    (one thread per row for the grid, one warp per row for the denser R-MAT);
    it follows the main kernel's recurrence (forced here with a variant)."""
    g = G.grid2d(33, 47) if name == "grid" else G.rmat(10, seed=4)
    assert g.m_directed + 8 * g.n <= 32768
    rp, col, w = g.row_ptr, g.col, None
    if weighted:
        hn = O.hec_heavy(rp, col, None, True, 5)
        vc, nc, _ = O.hec_map(hn, 5)
        rp, col, w = O.build_coarse(rp, col, None, vc, nc)
    n = rp.shape[0] - 1
    x0 = torch.from_numpy(np.random.default_rng(n).random(n)).cuda()
    args = (dev_u32(rp), dev_u32(col), None if w is None else dev_u32(w), x0, None, 1e-10, 3000)
    u_s, it_s, lam_s, _ = partitioner.power_iter(*args)
    monkeypatch.setenv("SGPB_PI_MODE", "rowp")
    u_m, it_m, lam_m, _ = partitioner.power_iter(*args)
    assert abs(it_s - it_m) <= 2
    assert abs(lam_s - lam_m) <= 1e-9 * abs(lam_m)
    u_o, it_o, lam_o = O.power_iter(rp, col, w, x0.cpu().numpy(), 1e-10, 3000)
    assert abs(it_s - it_o) <= max(2, it_o // 50) and abs(lam_s - lam_o) <= 1e-6 * abs(lam_o)
    if it_s == it_o:
        assert 1 - abs(float(np.dot(u_s.cpu().numpy(), u_o))) <= 1e-8


def test_power_iter_prolongation(partitioner):
    g = G.grid2d(40, 40)
    hn = O.hec_heavy(g.row_ptr, g.col, None, True, 3)
    vc, nc, _ = O.hec_map(hn, 3)
    xc = np.random.default_rng(1).random(nc)
    x0 = xc[vc]
    u_o, it_o, lam_o = O.power_iter(g.row_ptr, g.col, None, x0, 1e-10, 3000)
    u_g, it_g, lam_g, _ = partitioner.power_iter(dev_u32(g.row_ptr), dev_u32(g.col), None,
                                                 torch.from_numpy(xc).cuda(), dev_u32(vc), 1e-10, 3000)
    assert abs(lam_g - lam_o) <= 1e-6 * lam_o
    assert abs(it_g - it_o) <= max(2, it_o // 50)


def test_power_iter_grid_eigenvalue(partitioner):
    """Converged FP64 iteration on a 24x24 grid reaches the closed-form
    Fiedler value 2 - 2 cos(pi / 24) (independent check)."""
    g = G.grid2d(24, 24)
    x0 = np.random.default_rng(2).random(g.n)
    lam_exact = 2 - 2 * np.cos(np.pi / 24)
    _, it, lam, res = partitioner.power_iter(dev_u32(g.row_ptr), dev_u32(g.col), None, torch.from_numpy(x0).cuda(),
                                             None, 1e-15, 400000)
    assert abs(lam - lam_exact) / lam_exact < 1e-4


# ------------------------------------------------------------ whole path --
@pytest.mark.parametrize("name", ["grid64", "rmat12", "holes", "er3000"])
def test_partition_matches_oracle_hierarchy(partitioner, name):
    g = GRAPHS[name]()
    r = partitioner.partition(g, cutoff=50, tol=1e-10, rng_state=77)
    o = O.partition_graph(g.row_ptr, g.col, None, cutoff=50, tol=1e-10, rng_state=77)
    # integer hierarchy is bit-exact: the same level sizes
    assert r.levels == o["levels"]
    assert r.level_n == o["level_n"]
    assert r.rng_state == o["rng_state"]
    part = r.part
    assert part.sum() == g.n - g.n // 2 or part.sum() == g.n // 2 or abs(int(part.sum()) - g.n // 2) <= 1
    assert r.edgecut == O.edge_cut(g.row_ptr, g.col, part)
    # FP64 results: cut within 2% (+2 edges) of the oracle's
    assert abs(r.edgecut - o["edgecut"]) <= 0.02 * o["edgecut"] + 2
    assert abs(r.lam - o["lambda"]) <= 1e-6 * abs(o["lambda"]) + 1e-12


def test_partition_deterministic(partitioner):
    g = G.rmat(12, seed=5)
    a = partitioner.partition(g, rng_state=3)
    b = partitioner.partition(g, rng_state=3)
    assert np.array_equal(a.part, b.part) and a.edgecut == b.edgecut and a.level_iters == b.level_iters


MIXED_GRAPHS = {
    "rmat14": lambda: G.rmat(14, seed=9),
    "grid200": lambda: G.grid2d(200, 180),
    "holes": lambda: G.grid2d_holes(220, 200, 0.1, 4),
    "er40k": lambda: G.erdos_renyi(40000, 8.0, seed=3),
    "rgg100k": lambda: G.rgg3d(100000, seed=2),
    "chunglu_w": lambda: G.chung_lu(1 << 17, wmax=100, seed=1),
}


@pytest.mark.parametrize("name", sorted(MIXED_GRAPHS))
def test_mixed_precision_matches_fp64(partitioner, name):
    """Mixed precision (FP32 edge-difference SpMV arithmetic, FP64 iterate,
    shift, deflation, normalisation, dot and stopping test): the Fiedler value
    within 1e-6 relative of the FP64 path, the same hierarchy and iteration
    counts, the cut within 1%."""
    g = MIXED_GRAPHS[name]()
    a = partitioner.partition(g, rng_state=11, mixed=False)
    b = partitioner.partition(g, rng_state=11, mixed=True)
    assert abs(b.lam - a.lam) <= 1e-6 * abs(a.lam)
    assert b.level_n == a.level_n and b.level_iters == a.level_iters
    assert abs(b.edgecut - a.edgecut) <= 0.01 * a.edgecut
    assert b.edgecut == O.edge_cut(g.row_ptr, g.col, b.part)


def test_device_resident_input_and_output(partitioner):
    g = G.grid2d(50, 40)
    dg = {"row_ptr": dev_u32(g.row_ptr), "col": dev_u32(g.col)}
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    r = partitioner.partition(dg, rng_state=5, part_out=out)
    h = partitioner.partition(g, rng_state=5)
    assert np.array_equal(host_u32(out), h.part) and r.edgecut == h.edgecut


# ------------------------------------------------------------ sgpar.h API --
def test_sgpar_api_partition_graph():
    from ipdps_2021_graph_coarsening_b200 import api
    g = G.grid2d(40, 40)
    rng = api.PCG32(state=123, inc=1)
    part, cut = api.partition_graph(g, api.Config(), 0, rng)
    assert cut == O.edge_cut(g.row_ptr, g.col, part)
    assert part.sum() == g.n // 2
    assert rng.state != 123


def test_sgpar_api_compute_partition():
    from ipdps_2021_graph_coarsening_b200 import api
    g = G.grid2d(21, 23)
    ev = np.random.default_rng(4).standard_normal(g.n)
    p, c = api.compute_partition(ev, g)
    p_o, c_o = O.compute_partition(g.row_ptr, g.col, ev)
    assert np.array_equal(p, p_o) and c == c_o


def test_sgpar_api_use_partition():
    from ipdps_2021_graph_coarsening_b200 import api
    g = G.rmat(10, seed=2)
    part = (np.random.default_rng(1).random(g.n) < 0.5).astype(np.uint32)
    (a_rp, a_col), (b_rp, b_col) = O.use_partition(g.row_ptr, g.col, part)
    g1, g2 = api.use_partition(part, g)
    assert np.array_equal(g1.row_ptr, a_rp) and np.array_equal(g1.col, a_col)
    assert np.array_equal(g2.row_ptr, b_rp) and np.array_equal(g2.col, b_col)


# ------------------------------------------------------------ edge cases --
def test_graph_at_or_below_cutoff(partitioner):
    g = G.grid2d(5, 6)    # 30 vertices: no coarsening level
    r = partitioner.partition(g, cutoff=50, rng_state=1)
    o = O.partition_graph(g.row_ptr, g.col, None, cutoff=50, rng_state=1)
    assert r.levels == 1 == o["levels"]
    assert abs(r.edgecut - o["edgecut"]) <= 1


def test_isolated_vertices(partitioner):
    g = G.grid2d(20, 20)
    n = g.n + 7    # seven isolated vertices appended
    rp = np.concatenate([g.row_ptr, np.full(7, g.row_ptr[-1], np.uint32)])
    h = G.CSR(rp, g.col)
    for random_level in (True, False):
        hn_o = O.hec_heavy(h.row_ptr, h.col, None, random_level, 5)
        vc_o, nc_o, _ = O.hec_map(hn_o, 5)
        hn, vc, nc, _ = partitioner.hec(dev_u32(h.row_ptr), dev_u32(h.col), None, random_level, 5)
        assert nc == nc_o and np.array_equal(host_u32(vc), vc_o)
    r = partitioner.partition(h, rng_state=2)
    assert r.part.shape[0] == n


def test_malformed_graph_is_rejected(partitioner):
    from ipdps_2021_graph_coarsening_b200 import _lib as L
    g = G.grid2d(10, 10)
    bad = G.CSR(g.row_ptr.copy(), g.col.copy())
    bad.col[5] = 10_000
    with pytest.raises(L.SgparError) as e:
        partitioner.partition(bad)
    assert e.value.code == L.ERR_INVALID


def with_isolated(g, k, seed=0):
    """g plus k isolated vertices at random positions (rows without entries)."""
    rng = np.random.default_rng(seed)
    n2 = g.n + k
    old = np.sort(rng.choice(n2, g.n, replace=False)).astype(np.uint32)   # new id of each old vertex
    deg = np.zeros(n2, np.int64)
    deg[old] = np.diff(g.row_ptr).astype(np.int64)
    rp = np.zeros(n2 + 1, np.uint32)
    rp[1:] = np.cumsum(deg)
    col = np.empty(len(g.col), np.uint32)
    for i in range(g.n):
        col[rp[old[i]]:rp[old[i] + 1]] = old[g.col[g.row_ptr[i]:g.row_ptr[i + 1]]]
    return G.CSR(rp, col)


@pytest.mark.parametrize("name", ["er7k", "grid100", "er7k_isolated", "chunglu_w"])
@pytest.mark.parametrize("mixed", [False, True])
def test_power_iter_mid_size_cluster(partitioner, monkeypatch, name, mixed):
    """Mid-size levels (more than one block's shared memory, at most 2^17
    cost units) run on a cluster of blocks with the iterate in global memory
    and one cluster barrier per iteration: against the oracle, and against the
    cooperative kernel (SGPB_PI_MID=0), including rows without entries."""
    if name == "er7k":
        g = G.erdos_renyi(7500, 8.0, seed=7)
        rp, col, w = g.row_ptr, g.col, None
    elif name == "grid100":
        g = G.grid2d(100, 90)
        rp, col, w = g.row_ptr, g.col, None
    elif name == "er7k_isolated":
        g = with_isolated(G.erdos_renyi(7000, 8.0, seed=8), 200, seed=1)
        rp, col, w = g.row_ptr, g.col, None
    else:
        g = G.chung_lu(4000, wmax=50, seed=5)
        rp, col, w = g.row_ptr, g.col, g.w
    n = rp.shape[0] - 1
    assert 32768 < int(rp[-1]) + 8 * n <= (1 << 17)
    x0 = np.random.default_rng(n).random(n)
    args = (dev_u32(rp), dev_u32(col), None if w is None else dev_u32(w), torch.from_numpy(x0).cuda(), None,
            1e-10, 3000, mixed)
    u_c, it_c, lam_c, res_c = partitioner.power_iter(*args)
    u_o, it_o, lam_o = O.power_iter(rp, col, w, x0, 1e-10, 3000)
    assert abs(it_c - it_o) <= max(2, it_o // 50)
    assert abs(lam_c - lam_o) <= 1e-6 * abs(lam_o)
    if it_c == it_o:
        assert 1 - abs(float(np.dot(u_c.cpu().numpy(), u_o))) <= 1e-8
    u = u_c.cpu().numpy()
    assert abs(np.linalg.norm(u) - 1) < 1e-9 and abs(u.sum()) < 1e-8 * np.sqrt(n)
    monkeypatch.setenv("SGPB_PI_MID", "0")
    u_p, it_p, lam_p, _ = partitioner.power_iter(*args)
    # the two kernels add the FP32 partial sums of the mixed path in
    # different orders (isolated vertices make lambda ~1e-5: an absolute floor)
    assert abs(it_p - it_c) <= 2 and abs(lam_p - lam_c) <= (1e-8 if mixed else 1e-9) * abs(lam_c) + 1e-13
