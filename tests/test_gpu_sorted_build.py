"""The sorted coarse build of unit-weight levels (one radix sort of the packed
(coarse u, coarse v) keys, run lengths as weights) against the oracle's build
and the tiered build, bit for bit: a real HEC mapping of R-MAT 18 (above the
size where partitions take the sorted build), and mappings whose coarse count
is a power of two (the widest packed key next to the sentinel)."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O
from tests.test_gpu_parity import dev_u32, host_u32, host_u64

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def mapping(case):
    if case == "rmat18_hec":
        g = G.rmat(18, seed=2)
        hn = O.hec_heavy(g.row_ptr, g.col, None, True, 3)
        vc, nc, _ = O.hec_map(hn, 3)
        return g, np.asarray(vc, dtype=np.uint32), nc
    if case == "grid_mod64":
        g = G.grid2d(300, 300)
        return g, (np.arange(g.n) % 64).astype(np.uint32), 64
    g = G.erdos_renyi(20000, 8.0, seed=5)
    nc = 1 << 10
    vc = np.random.default_rng(1).integers(0, nc, g.n).astype(np.uint32)
    vc[:nc] = np.arange(nc, dtype=np.uint32)
    return g, vc, nc


def gpu_build(partitioner, g, vc, nc, wbytes):
    crp, ccol, cw = partitioner.build_coarse(dev_u32(g.row_ptr), dev_u32(g.col), None, dev_u32(vc), nc, wbytes)
    w = host_u32(cw) if wbytes == 4 else host_u64(cw)
    return host_u32(crp), host_u32(ccol), w.astype(np.uint64)


@pytest.mark.parametrize("case", ["rmat18_hec", "grid_mod64", "er_random_pow2"])
@pytest.mark.parametrize("wbytes", [4, 8])
def test_sorted_build_matches_oracle_and_tiered(partitioner, monkeypatch, case, wbytes):
    g, vc, nc = mapping(case)
    want = O.build_coarse(g.row_ptr, g.col, None, vc, nc)
    monkeypatch.setenv("SGPB_BUILD_SORTED", "1")
    got = gpu_build(partitioner, g, vc, nc, wbytes)
    monkeypatch.setenv("SGPB_BUILD_SORTED", "0")
    tiered = gpu_build(partitioner, g, vc, nc, wbytes)
    for a, b, c in zip(got, tiered, want):
        assert np.array_equal(a, c) and np.array_equal(b, c)


def test_partition_same_with_either_build(partitioner, monkeypatch):
    """A whole partition of a large unit-weight graph gives the same
    hierarchy, iterations and partition with the sorted build (forced) and
    the default tiered build."""
    g = G.rmat(18, seed=4)
    assert g.m_directed >= 1 << 22
    monkeypatch.setenv("SGPB_BUILD_SORTED", "1")
    a = partitioner.partition(g, rng_state=6)
    monkeypatch.delenv("SGPB_BUILD_SORTED")
    b = partitioner.partition(g, rng_state=6)
    assert a.level_n == b.level_n and a.level_m == b.level_m and a.level_iters == b.level_iters
    assert np.array_equal(np.asarray(a.part), np.asarray(b.part)) and a.edgecut == b.edgecut
