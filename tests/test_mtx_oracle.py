"""The CPU restatement of the MatrixMarket converter (oracle/mtx_oracle.py)
pinned byte for byte against the reference's own converters
(cmg/mtx2csr.cpp and cmg/mtx2csr_large.cpp, built from their sources into
oracle/_ref by oracle/Makefile) on every case with defined behaviour, and its
rejection of the malformed cases."""
import pytest

from oracle import mtx_oracle as M
from tests import mtx_cases as MC

VALID = MC.valid_cases()
INVALID = MC.invalid_cases()


@pytest.mark.parametrize("name", sorted(VALID))
def test_oracle_matches_reference_converter(name, tmp_path):
    if not MC.reference_available(4):
        pytest.skip("reference converter not built (oracle/Makefile)")
    rp, col, info = M.convert(VALID[name])
    assert M.csr_bytes(rp, col) == MC.run_reference(VALID[name], str(tmp_path))


@pytest.mark.parametrize("name", ["holes_dups_isolated", "bipartite_40x70", "tie_two_triangles", "empty_size"])
def test_oracle_matches_large_converter(name, tmp_path):
    if not MC.reference_available(8):
        pytest.skip("reference converter not built (oracle/Makefile)")
    rp, col, _ = M.convert(VALID[name])
    assert M.csr_bytes(rp, col, 8) == MC.run_reference(VALID[name], str(tmp_path), 8)


@pytest.mark.parametrize("name", sorted(INVALID))
def test_oracle_rejects(name):
    with pytest.raises(M.MtxError):
        M.convert(INVALID[name])


def test_round_trip_of_a_clean_graph():
    """A connected graph without duplicates comes back unchanged, whatever
    the line order, duplicates, values and isolated vertices of its file."""
    from ipdps_2021_graph_coarsening_b200 import graphs as G
    g = G.rmat(11, seed=6)
    for kw in ({"seed": 1}, {"seed": 2, "dup_frac": 0.5, "extra_vertices": 100, "field": "real"},
               {"symmetry": "general", "seed": 3}):
        rp, col, info = M.convert(G.mtx_of(g, **kw))
        assert (rp == g.row_ptr).all() and (col == g.col).all()
        assert info["n"] == g.n and info["components"] == 1 + kw.get("extra_vertices", 0)
