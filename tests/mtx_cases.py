"""MatrixMarket inputs shared by the converter tests: the cases the
reference's converter (cmg/mtx2csr.cpp) handles with defined behaviour, and
the malformed ones the device path must reject."""
from __future__ import annotations

import os
import subprocess

import numpy as np

from ipdps_2021_graph_coarsening_b200 import graphs as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = {4: os.path.join(ROOT, "oracle", "_ref", "mtx2csr"), 8: os.path.join(ROOT, "oracle", "_ref", "mtx2csr_large")}

BANNER = b"%%MatrixMarket matrix coordinate pattern symmetric\n"
GENERAL = b"%%MatrixMarket matrix coordinate pattern general\n"


def _tri(a, b, c):
    return f"{a} {b}\n{b} {c}\n{c} {a}\n".encode()


def valid_cases() -> dict[str, bytes]:
    """name -> text, all with defined behaviour in the reference."""
    c = {}
    c["grid_sym_shuffled"] = G.mtx_of(G.grid2d(30, 20), seed=3)
    c["grid_sym_rows"] = G.mtx_of(G.grid2d(17, 9), seed=None)
    c["holes_dups_isolated"] = G.mtx_of(G.grid2d_holes(40, 40, 0.1, 2), seed=5, dup_frac=0.3, extra_vertices=7)
    c["rmat10_general_real"] = G.mtx_of(G.rmat(10, seed=4), symmetry="general", field="real", seed=1)
    c["er_integer_crlf"] = G.mtx_of(G.erdos_renyi(700, 3.0, seed=2), field="integer", seed=9, crlf=True,
                                    comments=["generated", " second comment"])
    # general square, one direction only: read as A + A^T
    rng = np.random.default_rng(11)
    u = rng.integers(0, 300, 1500)
    v = rng.integers(0, 300, 1500)
    c["general_square_asym_loops"] = G.mtx_text(u, v, 300, 300, symmetry="general")
    # general rectangular: bipartite, rows after the columns
    u = rng.integers(0, 40, 200)
    v = rng.integers(0, 70, 200)
    c["bipartite_40x70"] = G.mtx_text(u, v, 40, 70, symmetry="general", field="real")
    c["bipartite_70x40"] = G.mtx_text(v, u, 70, 40, symmetry="general")
    # self loops and duplicates in a symmetric file
    c["loops_dups"] = BANNER + b"6 6 9\n1 1\n2 1\n2 1\n3 2\n3 3\n4 3\n1 2\n6 5\n5 5\n"
    # two equally large components: the one with the smaller vertex wins
    c["tie_two_triangles"] = BANNER + b"7 7 6\n" + _tri(5, 6, 7) + _tri(2, 3, 4)
    c["tie_reverse"] = BANNER + b"7 7 6\n" + _tri(1, 2, 3) + _tri(5, 6, 7)
    c["larger_second"] = BANNER + b"9 9 7\n" + _tri(1, 2, 3) + b"5 6\n6 7\n7 8\n8 9\n"
    # comments between entries, blank-free, no final newline
    c["comments_inside_no_eol"] = BANNER + b"% head\n4 4 3\n2 1\n% mid\n3 2\n%\n4 3"
    c["plus_signs_tabs"] = BANNER + b"4 4 3\n+2\t1\n 3 +2 \r\n4\t\t3 0.5e3\n"
    # all vertices isolated: the first one alone
    c["no_edges"] = BANNER + b"5 5 0\n"
    c["only_loops"] = BANNER + b"3 3 3\n1 1\n2 2\n3 3\n"
    c["empty_size"] = BANNER + b"0 0 0\n"
    c["banner_only"] = BANNER
    c["one_edge"] = BANNER + b"2 2 1\n2 1\n"
    c["two_comment_lines_before_size"] = b"%%MatrixMarket matrix coordinate real general\n%a\n%b\n3 3 2\n1 2 1.0\n3 2 2.0\n"
    c["later_banner_harmless"] = BANNER + b"3 3 2\n2 1\n%%MatrixMarket matrix coordinate pattern symmetric\n3 2\n"
    return c


def invalid_cases() -> dict[str, bytes]:
    """name -> text the reference handles with undefined behaviour or an
    exit; both the oracle and the device path must reject them."""
    return {
        "array_format": b"%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",
        "symmetric_not_square": BANNER + b"3 4 1\n1 1\n",
        "id_zero": BANNER + b"3 3 1\n0 1\n",
        "id_beyond_size": BANNER + b"3 3 2\n2 1\n4 1\n",
        "bipartite_row_beyond": GENERAL + b"2 5 1\n3 1\n",
        "one_number": BANNER + b"3 3 1\n2\n",
        "negative_id": BANNER + b"3 3 1\n-2 1\n",
        "letters": BANNER + b"3 3 1\nx y\n",
        "bad_size_line": BANNER + b"three 3 3\n1 2\n",
        "later_banner_not_coordinate": BANNER + b"3 3 2\n2 1\n%%MatrixMarket matrix array real\n3 2\n",
        "later_banner_general": BANNER + b"3 3 2\n2 1\n%%MatrixMarket matrix coordinate pattern general\n3 2\n",
    }


def run_reference(text: bytes, tmpdir: str, id_bytes: int = 4) -> bytes:
    """The reference converter's output file for `text`."""
    src = os.path.join(tmpdir, "in.mtx")
    dst = os.path.join(tmpdir, "out.csr")
    with open(src, "wb") as f:
        f.write(text)
    r = subprocess.run([REF_BIN[id_bytes], src, dst], capture_output=True, timeout=120)
    if r.returncode != 0:
        raise RuntimeError(f"reference converter failed: {r.stdout[-400:]!r} {r.stderr[-400:]!r}")
    with open(dst, "rb") as f:
        return f.read()


def reference_available(id_bytes: int = 4) -> bool:
    return os.path.exists(REF_BIN[id_bytes])
