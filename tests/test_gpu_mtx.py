"""The device MatrixMarket converter (sgp_b200_mtx_read / _parse / mtx2csr)
against the reference's own converter binaries (oracle/_ref, built from
cmg/mtx2csr.cpp and cmg/mtx2csr_large.cpp) and the CPU restatement
(oracle/mtx_oracle.py): output files byte for byte, statistics exactly, the
malformed inputs rejected, and at sizes beyond the oracle the round trip of a
clean graph through a shuffled file with duplicates and isolated vertices."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import mtx_oracle as M
from tests import mtx_cases as MC

pytestmark = pytest.mark.gpu

VALID = MC.valid_cases()
INVALID = MC.invalid_cases()


def expected(text, tmp_path, id_bytes=4):
    """The reference binary's output where it is built, else the oracle's."""
    rp, col, info = M.convert(text)
    want = M.csr_bytes(rp, col, id_bytes)
    if MC.reference_available(id_bytes):
        assert MC.run_reference(text, str(tmp_path), id_bytes) == want
    return want, info


def check_info(info, oinfo):
    for k in ("n_all", "m_all", "components", "n", "m", "lines", "bipartite", "rows", "cols"):
        assert info[k] == oinfo[k], k


@pytest.mark.parametrize("name", sorted(VALID))
def test_text_matches_reference(partitioner, name, tmp_path):
    want, oinfo = expected(VALID[name], tmp_path)
    g, info = partitioner.mtx_read(VALID[name])
    assert M.csr_bytes(g.row_ptr, g.col) == want
    check_info(info, oinfo)


@pytest.mark.parametrize("name", ["holes_dups_isolated", "bipartite_70x40", "er_integer_crlf", "banner_only"])
@pytest.mark.parametrize("id_bytes", [4, 8])
def test_mtx2csr_command_file(partitioner, name, id_bytes, tmp_path):
    src, dst = tmp_path / "g.mtx", tmp_path / "g.csr"
    src.write_bytes(VALID[name])
    want, oinfo = expected(VALID[name], tmp_path, id_bytes)
    info = partitioner.mtx2csr(str(src), str(dst), id_bytes)
    assert dst.read_bytes() == want
    check_info(info, oinfo)


def test_file_and_device_sources_agree(partitioner, tmp_path):
    torch = pytest.importorskip("torch")
    text = G.mtx_of(G.grid2d_holes(90, 70, 0.12, 3), seed=2, dup_frac=0.2, extra_vertices=11)
    src = tmp_path / "h.mtx"
    src.write_bytes(text)
    a, ia = partitioner.mtx_read(str(src))
    b, ib = partitioner.mtx_read(text)
    dtext = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    (rp, col), ic = partitioner.mtx_read(dtext, device_out=True)
    rp, col = rp.cpu().numpy().view(np.uint32), col.cpu().numpy().view(np.uint32)
    for x in (b,):
        assert np.array_equal(x.row_ptr, a.row_ptr) and np.array_equal(x.col, a.col)
    assert np.array_equal(rp, a.row_ptr) and np.array_equal(col, a.col)
    assert ia["m"] == ib["m"] == ic["m"] and ia["components"] == ic["components"] == 12


@pytest.mark.parametrize("name", sorted(INVALID))
def test_malformed_rejected(partitioner, name):
    with pytest.raises(L.SgparError) as e:
        partitioner.mtx_read(INVALID[name])
    assert e.value.code == L.ERR_INVALID


def test_error_names_the_line(partitioner):
    text = MC.BANNER + b"% c\n5 5 3\n2 1\n3 2\n6 1\n"
    with pytest.raises(L.SgparError, match="line 6"):
        partitioner.mtx_read(text)


def test_missing_file(partitioner, tmp_path):
    with pytest.raises(L.SgparError, match="could not open"):
        partitioner.mtx_read(str(tmp_path / "none.mtx"))


@pytest.mark.parametrize("case", ["rmat16_general_dups", "chunglu_hubs", "star", "many_components", "rmat15_rows"])
def test_larger_inputs_match_oracle(partitioner, case):
    """Sizes where every dedupe tier (warp, block, dense) and the union-find
    see real work; hubs hit the aggregated atomics and the dense tier."""
    if case == "rmat16_general_dups":
        text = G.mtx_of(G.rmat(16, seed=2), symmetry="general", seed=4, dup_frac=0.3, extra_vertices=500)
    elif case == "chunglu_hubs":
        text = G.mtx_of(G.chung_lu(60000, wmax=0, seed=3), seed=1, dup_frac=0.1)
    elif case == "star":
        n = 20000
        text = G.mtx_text(np.arange(1, n), np.zeros(n - 1, np.int64), n, n)
    elif case == "many_components":
        rng = np.random.default_rng(8)
        n = 50000   # sparse random graph below the giant-component threshold
        u, v = rng.integers(0, n, 20000), rng.integers(0, n, 20000)
        text = G.mtx_text(u, v, n, n, symmetry="general")
    else:
        text = G.mtx_of(G.rmat(15, seed=9), seed=None)   # sorted by row: ids repeat within warps
    rp, col, oinfo = M.convert(text)
    g, info = partitioner.mtx_read(text)
    assert np.array_equal(g.row_ptr, rp) and np.array_equal(g.col, col)
    check_info(info, oinfo)


@pytest.mark.parametrize("scale", [18, 20])
def test_round_trip_at_size(partitioner, scale):
    """CSR -> shuffled MatrixMarket with duplicates and isolated vertices ->
    device converter gives the graph back exactly (a clean connected graph is
    its own largest component)."""
    g = G.rmat(scale, seed=1)
    extra = 1000
    text = G.mtx_of(g, seed=7, dup_frac=0.1, extra_vertices=extra, field="real")
    out, info = partitioner.mtx_read(text)
    assert np.array_equal(out.row_ptr, g.row_ptr) and np.array_equal(out.col, g.col)
    assert info["components"] == 1 + extra and info["n_all"] == g.n + extra and info["n"] == g.n
    assert info["m_all"] == info["m"] == g.m_directed


def test_converter_feeds_the_partitioner(partitioner):
    """mtx text -> device CSR -> partition, with no host round trip of the
    graph, equals partitioning the host copy."""
    g = G.grid2d_holes(120, 100, 0.1, 4)
    text = G.mtx_of(g, seed=3, extra_vertices=5)
    (rp, col), _ = partitioner.mtx_read(text, device_out=True)
    r_dev = partitioner.partition({"row_ptr": rp, "col": col}, rng_state=5)
    host, _ = partitioner.mtx_read(text)
    r_host = partitioner.partition(host, rng_state=5)
    assert np.array_equal(r_dev.part, r_host.part) and r_dev.edgecut == r_host.edgecut


def test_command_line_module(tmp_path):
    """python -m ipdps_2021_graph_coarsening_b200.mtx2csr writes the same file."""
    import subprocess
    import sys
    src, dst = tmp_path / "g.mtx", tmp_path / "g.csr"
    text = VALID["holes_dups_isolated"]
    src.write_bytes(text)
    want, _ = expected(text, tmp_path)
    r = subprocess.run([sys.executable, "-m", "ipdps_2021_graph_coarsening_b200.mtx2csr", str(src), str(dst)],
                       capture_output=True, text=True, cwd=MC.ROOT)
    assert r.returncode == 0, r.stderr
    assert dst.read_bytes() == want and "components" in r.stdout
