"""sgp_b200_split_noalloc, the split entry point that allocates nothing.

Some callers cannot allocate device memory when they need the split: a host
application that routes every device allocation through its own pool, code
running inside an out-of-memory handler, or a plug-in whose host forbids
allocation calls.  For them the library keeps a fixed scratch array and this
entry point uses only that.  Its results must equal those of the allocating
entry point sgp_b200_split -- the split and the cut are integer work, so the
comparison is exact -- including on consecutive calls that reuse the shared
scratch.  This file is collected last so that a stop at its first failure
still leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import graphs as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev_u32(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def split_noalloc(g, ev):
    """One call through the C ABI on torch's current stream."""
    rp, col = dev_u32(g.row_ptr), dev_u32(g.col)
    evd = torch.from_numpy(np.ascontiguousarray(ev, dtype=np.float64)).cuda()
    part = torch.full((g.n,), -1, dtype=torch.int32, device="cuda")
    res = torch.zeros(2, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.lib().sgp_b200_split_noalloc(ctypes.c_void_p(stream), g.n, rp.data_ptr(), col.data_ptr(),
                                         evd.data_ptr(), part.data_ptr(), res.data_ptr())
    torch.cuda.synchronize()
    return rc, part.cpu().numpy().view(np.uint32), int(res[0].item()), int(res[1].item())


def split_allocating(partitioner, g, ev):
    part, cut = partitioner.split(dev_u32(g.row_ptr), dev_u32(g.col),
                                  torch.from_numpy(np.ascontiguousarray(ev, dtype=np.float64)).cuda())
    return part.cpu().numpy().view(np.uint32), cut


def vector(n, seed, ties):
    ev = np.random.default_rng(seed).standard_normal(n)
    if ties:
        ev = np.round(ev, 1)
        ev[::7] = 0.0
    return ev


def test_noalloc_matches_split_on_consecutive_calls(partitioner):
    cases = [(G.grid2d(33, 47), vector(33 * 47, 1, True)),       # odd n: the sweep vertex
             (G.rmat(12, seed=4), None),                          # a different size in between
             (G.grid2d(33, 47), vector(33 * 47, 1, True))]        # the first case again
    cases[1] = (cases[1][0], vector(cases[1][0].n, 2, False))
    outs = []
    for g, ev in cases:
        rc, part, cut, p0 = split_noalloc(g, ev)
        assert rc == L.OK, L.last_error()
        ref_part, ref_cut = split_allocating(partitioner, g, ev)
        assert cut == ref_cut
        assert np.array_equal(part, ref_part)
        assert p0 == int((part == 0).sum())
        outs.append((part, cut))
    assert np.array_equal(outs[0][0], outs[2][0]) and outs[0][1] == outs[2][1]


def path_graph(n):
    """A path of n vertices (n = 1: a single isolated vertex)."""
    deg = np.full(n, 2, np.uint32)
    if n == 1:
        deg[0] = 0
    else:
        deg[0] = deg[-1] = 1
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum(deg)
    col = np.empty(int(rp[-1]), np.uint32)
    i = np.arange(n, dtype=np.uint32)
    left = rp[1:n] if n > 1 else np.zeros(0, np.uint32)    # slot of the entry i -> i - 1 in rows 1..n-1
    col[left] = i[1:] - 1
    right = rp[:n - 1] + (np.arange(n - 1) > 0)             # slot of the entry i -> i + 1 in rows 0..n-2
    col[right] = i[:n - 1] + 1
    return G.CSR(rp, col)


@pytest.mark.parametrize("n", [1, 1 << 20])
def test_noalloc_smallest_and_largest_inputs(partitioner, n):
    """One vertex (the sweep vertex is the only vertex) and exactly
    SGP_B200_NOALLOC_MAX_N vertices, which fills the keys region up to the
    histograms; each twice in a row, equal to the allocating split."""
    g = path_graph(n)
    ev = vector(n, 3, True)
    ref_part, ref_cut = split_allocating(partitioner, g, ev)
    for _ in range(2):
        rc, part, cut, p0 = split_noalloc(g, ev)
        assert rc == L.OK, L.last_error()
        assert cut == ref_cut and np.array_equal(part, ref_part)
        assert p0 == int((part == 0).sum())


def test_noalloc_rejects_sizes_beyond_its_scratch():
    small = torch.zeros(4, dtype=torch.int64, device="cuda")
    p = small.data_ptr()
    rc = L.lib().sgp_b200_split_noalloc(None, (1 << 20) + 1, p, p, p, p, p)
    assert rc == L.ERR_TOO_LARGE
    assert "vertices" in L.last_error()
