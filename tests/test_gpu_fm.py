"""FM refinement on the device (fm.cu) against the oracle's restatement of
the same pass (oracle/sgpar_oracle.c orc_fm_refine): partitions, cuts, pass
and move counts bit for bit from spectral, random and skewed starting
bisections, and the whole path with fm_passes."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = {
    "grid": lambda: G.grid2d(120, 90),
    "holes": lambda: G.grid2d_holes(150, 120, 0.1, 2),
    "er": lambda: G.erdos_renyi(20000, 5.0, seed=3),
    "rmat": lambda: G.rmat(14, seed=2),
    "rgg": lambda: G.rgg3d(40000, seed=1),
    "chunglu": lambda: G.chung_lu(30000, wmax=0, seed=4),
}


def starts(g):
    rng = np.random.default_rng(11)
    spectral = O.partition_graph(g.row_ptr, g.col, None, rng_state=5)["part"]
    rand = (rng.permutation(g.n) < g.n // 2).astype(np.uint32)
    skew = (rng.permutation(g.n) < int(0.6 * g.n)).astype(np.uint32)   # |d| = 0.2 n: target |d| / 10
    return {"spectral": spectral, "random": rand, "skewed": skew}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fm_bit_exact(partitioner, name):
    g = CASES[name]()
    rp = torch.from_numpy(g.row_ptr.view(np.int32)).cuda()
    col = torch.from_numpy(g.col.view(np.int32)).cuda()
    for label, p0 in starts(g).items():
        pd = torch.from_numpy(p0.astype(np.uint32).view(np.int32)).cuda()
        cut, passes, moves = partitioner.fm_refine(rp, col, pd, 16)
        op, oc, opasses, omoves = O.fm_refine(g.row_ptr, g.col, None, p0, 16)
        got = pd.cpu().numpy().view(np.uint32)
        assert (passes, moves) == (opasses, omoves), label
        assert np.array_equal(got, op) and cut == oc == O.edge_cut(g.row_ptr, g.col, got), label


@pytest.mark.parametrize("name", ["holes", "rmat", "rgg"])
def test_partition_with_fm(partitioner, name):
    g = CASES[name]()
    base = partitioner.partition(g, rng_state=3)
    r = partitioner.partition(g, rng_state=3, fm_passes=16)
    cut = O.edge_cut(g.row_ptr, g.col, r.part)
    assert r.edgecut == cut <= base.edgecut
    assert r.part0_size == int((r.part == 0).sum())
    assert abs(2 * r.part0_size - g.n) <= 20 + 1
    # the same passes from the same split on the oracle
    op, oc, _, _ = O.fm_refine(g.row_ptr, g.col, None, base.part, 16)
    assert np.array_equal(r.part, op) and r.edgecut == oc
