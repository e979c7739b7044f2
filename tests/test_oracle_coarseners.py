"""The oracle's restatements of the reference's alternative coarseners
(oracle/sgpar_oracle.c: orc_match_map, orc_set_map) checked against the
invariants that the reference algorithms guarantee whatever their random keys
and thread timing (cmg/heuristics.h):

  MATCH (:1584-1740)  aggregates of one or two vertices, pairs are edges, and
                      no two singletons are adjacent (a vertex leaves the
                      rounds only when all its neighbours are matched)
  MIS2  (:8-80, :218-310)  roots pairwise at distance >= 3, every vertex in
                      the aggregate of a root at distance <= 2, one root per
                      aggregate
  GOSH  (:81-216, :312-365)  one set vertex per aggregate, every other
                      vertex adjacent to its aggregate's set vertex, which has
                      the largest degree among its set neighbours; no two set
                      vertices adjacent unless both exceed the mean degree

and the whole path with each coarsener producing a valid bisection."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O


def cases():
    return {
        "grid": G.grid2d(40, 30),
        "holes": G.grid2d_holes(50, 40, 0.15, 3),
        "rmat": G.rmat(11, seed=5),
        "chunglu_w": G.chung_lu(3000, wmax=50, seed=2),
        "er": G.erdos_renyi(2000, 4.0, seed=7),
    }


CASES = cases()


def rows(g):
    return np.repeat(np.arange(g.n), np.diff(g.row_ptr).astype(np.int64))


def members(vc, nc):
    order = np.argsort(vc, kind="stable")
    bounds = np.searchsorted(vc[order], np.arange(nc + 1))
    return [order[bounds[c]:bounds[c + 1]] for c in range(nc)]


def bfs_dist(g, src, limit=3):
    dist = {int(src): 0}
    frontier = [int(src)]
    for d in range(1, limit + 1):
        nxt = []
        for u in frontier:
            for v in g.col[g.row_ptr[u]:g.row_ptr[u + 1]]:
                v = int(v)
                if v not in dist:
                    dist[v] = d
                    nxt.append(v)
        frontier = nxt
    return dist


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("random_level", [True, False])
def test_match_is_a_maximal_matching(name, random_level):
    g = CASES[name]
    vc, nc, rounds = O.match_map(g.row_ptr, g.col, g.w, random_level, seed=0x1234)
    assert sorted(set(vc.tolist())) == list(range(nc))
    sizes = np.bincount(vc, minlength=nc)
    assert sizes.max() <= 2 and rounds >= 1
    # pairs are edges
    r = rows(g)
    same = vc[r] == vc[g.col]
    paired = np.zeros(g.n, bool)
    paired[r[same]] = True
    assert np.array_equal(paired, sizes[vc] == 2)
    # no two adjacent singletons
    single = sizes[vc] == 1
    assert not np.any(single[r] & single[g.col])


@pytest.mark.parametrize("name", ["grid", "holes", "rmat", "er"])
def test_mis2_aggregates(name):
    g = CASES[name]
    vc, nc, its = O.set_map(g.row_ptr, g.col, False, seed=99)
    assert sorted(set(vc.tolist())) == list(range(nc)) and its >= 1
    # roots: the vertices numbered in ascending order are the first member of
    # each aggregate that is adjacent to all its distance-1 members; recover
    # them as the unique member within distance 2 of all others
    r = rows(g)
    for agg in members(vc, nc)[:400]:
        ok = False
        for cand in agg:
            d = bfs_dist(g, cand, 2)
            if all(int(x) in d for x in agg):
                ok = True
                break
        assert ok, "aggregate not within distance 2 of one vertex"
    # distance-2 independence of roots: each aggregate has one root and roots
    # of different aggregates are not within distance 2 (the root of every
    # aggregate is its member whose neighbours are all in it)
    roots = []
    for agg in members(vc, nc):
        s = set(agg.tolist())
        rs = [u for u in agg if all(int(v) in s for v in g.col[g.row_ptr[u]:g.row_ptr[u + 1]])]
        assert rs, "no root whose neighbourhood lies inside its aggregate"
        roots.append(rs[0])
    sample = roots[:: max(1, len(roots) // 200)]
    rootset = set(int(x) for x in roots)
    for rt in sample:
        d = bfs_dist(g, rt, 2)
        assert not any(v in rootset and v != rt for v in d), "two roots within distance 2"


@pytest.mark.parametrize("name", sorted(CASES))
def test_gosh_aggregates(name):
    g = CASES[name]
    vc, nc, its = O.set_map(g.row_ptr, g.col, True, seed=5)
    assert sorted(set(vc.tolist())) == list(range(nc))
    deg = np.diff(g.row_ptr).astype(np.int64)
    thr = int(g.row_ptr[-1]) // g.n
    centre = {}
    for c, agg in enumerate(members(vc, nc)):
        # the centre is adjacent to every other member
        s = set(agg.tolist())
        cands = [u for u in agg
                 if all(int(x) == u or int(x) in set(g.col[g.row_ptr[u]:g.row_ptr[u + 1]].tolist()) for x in agg)]
        assert cands, "aggregate without a centre adjacent to all members"
        centre[c] = cands
    # set vertices: exactly one per aggregate; adjacent set vertices only
    # when both exceed the mean degree (those edges are ignored)
    r = rows(g)
    is_c = np.zeros(g.n, bool)
    for c, cands in centre.items():
        if len(cands) == 1:
            is_c[cands[0]] = True
    both = is_c[r] & is_c[g.col]
    assert np.all((deg[r[both]] > thr) & (deg[g.col[both]] > thr))


@pytest.mark.parametrize("coarsener", [1, 2, 3, 1 | 32, 16])
def test_whole_path_with_each_coarsener(coarsener):
    g = G.grid2d_holes(60, 50, 0.1, 4)
    o = O.partition_graph(g.row_ptr, g.col, None, rng_state=3, coarsener=coarsener)
    assert int((o["part"] == 0).sum()) in (g.n // 2, (g.n + 1) // 2)
    r = rows(g)
    assert o["edgecut"] == int((o["part"][r] != o["part"][g.col]).sum()) // 2
    if coarsener == 16:
        assert o["levels"] == 1
    else:
        # levels shrink; the coarsest may stay above the cutoff when the next
        # one fell below 10 vertices and was dropped (coarsen_kokkos.h:1226)
        ln = o["level_n"]
        assert o["levels"] > 1 and all(a > b for a, b in zip(ln, ln[1:]))


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("random_level", [True, False])
def test_hec_v3_aggregates(name, random_level):
    """heuristics.h:766-834: roots are the smaller ends of mutual heavy pairs
    and the other heavy-neighbour targets; every vertex that is neither joins
    its heavy neighbour's aggregate, and a mutual pair shares one."""
    g = CASES[name]
    seed = 0x5151
    hn = O.hec_heavy(g.row_ptr, g.col, g.w, random_level, seed)
    vc, nc = O.hec_v3_map(g.row_ptr, g.col, g.w, random_level, seed)
    assert sorted(set(vc.tolist())) == list(range(nc))
    n = g.n
    targeted = np.zeros(n, bool)
    targeted[hn] = True
    mutual = hn[hn] == np.arange(n)
    plain = ~targeted & ~mutual
    assert np.all(vc[plain] == vc[hn[plain]])
    assert np.all(vc[mutual] == vc[hn[mutual]])
    roots = (mutual & (np.arange(n) < hn)) | (targeted & ~mutual)
    assert nc == int(roots.sum())


@pytest.mark.parametrize("name", sorted(CASES))
def test_gosh_v2_aggregates(name):
    """heuristics.h:444-560: vertices above max(nnz / n, 50) degree are
    roots of their own aggregates, every vertex ends in an aggregate with a
    neighbour or alone, and the mapping is onto."""
    g = CASES[name]
    vc, nc = O.gosh_v2_map(g.row_ptr, g.col, g.w, seed=31)
    assert sorted(set(vc.tolist())) == list(range(nc))
    deg = np.diff(g.row_ptr).astype(np.int64)
    thr = max(int(g.row_ptr[-1]) // g.n, 50)
    big = np.flatnonzero(deg > thr)
    assert len(set(vc[big].tolist())) == len(big)   # one root per aggregate
    r = rows(g)
    same = np.zeros(g.n, bool)
    same[r[vc[r] == vc[g.col]]] = True
    sizes = np.bincount(vc, minlength=nc)
    assert np.all(same | (sizes[vc] == 1))
