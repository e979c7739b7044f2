"""Generate tests/golden/golden.npz from the reference's own code.

Run here (where the reference sources are compiled into oracle/_ref):

    python tests/golden/make_golden.py

Every expected output below is produced by the reference's serial build of
cmg/sgpar.h (oracle/ref_harness.cpp); the inputs are seeded.  The dedupe
known-answer test is the one in cmg/tests.cpp:7-56 (expected weights
{37, 24, 56, 41, 37} for destinations 0..4).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import bindings as O  # noqa: E402
from ipdps_2021_graph_coarsening_b200 import graphs as G  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")


def symmetric_weights(rp, col, seed, lo=1, hi=9):
    """Random symmetric integer weights for an unweighted symmetric CSR."""
    n = rp.shape[0] - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp).astype(np.int64))
    a = np.minimum(rows, col.astype(np.int64))
    b = np.maximum(rows, col.astype(np.int64))
    h = (a * 1000003 + b * 7919 + seed * 104729) % (hi - lo + 1)
    return (h + lo).astype(np.uint32)


def main() -> None:
    d = {}
    # -- dedupe known-answer test (cmg/tests.cpp:7-56)
    offs = np.array([0, 10, 15, 25, 31], np.uint32)
    dests = np.zeros(31, np.uint32)
    wgts = np.zeros(31, np.uint32)
    for i in range(4):
        for j in range(offs[i], offs[i + 1]):
            dests[j] = j - offs[i]
            wgts[j] = j
    dests[16:25] = [2, 4, 3, 2, 4, 2, 0, 3, 1]
    d["kat_dests"], d["kat_wgts"] = dests.copy(), wgts.copy()
    d["kat_expected"] = np.array([15 + 22, 24, 16 + 19 + 21, 18 + 23, 17 + 20], np.uint64)
    for kind in ("heap", "hashmap"):
        dd, ww = dests.copy(), wgts.copy()
        eps = np.zeros(5, np.uint32)
        import ctypes
        tot = ctypes.c_uint64(0)
        fn = getattr(O.ref(), f"ref_{kind}_deduplicate")
        fn(offs[2:].copy(), dd, ww, eps[2:].copy(), ctypes.byref(tot))
        m = int(tot.value)
        order = np.argsort(dd[15:15 + m], kind="stable")
        d[f"kat_{kind}_dst"] = dd[15:15 + m][order]
        d[f"kat_{kind}_w"] = ww[15:15 + m][order].astype(np.uint64)

    rng = np.random.default_rng(20210517)
    # -- power iteration, finest-level form (unit weights), grid 16x16
    g = G.grid2d(16, 16)
    u0 = rng.random(g.n)
    d["pi_grid_rp"], d["pi_grid_col"], d["pi_grid_u0"] = g.row_ptr, g.col, u0
    d["pi_grid_out"] = O.ref_power_iter(g.row_ptr, g.col, None, u0, True, 1e-10)
    # -- power iteration, coarse-level form (weights), ER graph
    e = G.erdos_renyi(300, 6.0, seed=5)
    w = symmetric_weights(e.row_ptr, e.col, 3)
    u1 = rng.random(e.n)
    d["pi_er_rp"], d["pi_er_col"], d["pi_er_w"], d["pi_er_u0"] = e.row_ptr, e.col, w, u1
    d["pi_er_out"] = O.ref_power_iter(e.row_ptr, e.col, w, u1, False, 1e-10)
    # -- median split, odd n, with ties in the vector
    g2 = G.grid2d(15, 17)
    ev = np.round(rng.standard_normal(g2.n), 2)
    d["split_rp"], d["split_col"], d["split_ev"] = g2.row_ptr, g2.col, ev
    p, c = O.ref_compute_partition(g2.row_ptr, g2.col, ev)
    d["split_part"], d["split_cut"] = p, np.array([c], np.uint64)
    # -- coarse build on a given mapping: R-MAT scale 10, two levels
    r = G.rmat(10, seed=7)
    hn = O.hec_heavy(r.row_ptr, r.col, None, True, 99)
    vc, nc, _ = O.hec_map(hn, 99)
    crp, ccol, cw, _ = O.ref_build_coarse(r.row_ptr, r.col, None, vc, nc, 1)
    d["build_rp"], d["build_col"], d["build_vcmap"] = r.row_ptr, r.col, vc
    d["build_nc"] = np.array([nc], np.uint32)
    d["build_out_rp"], d["build_out_col"], d["build_out_w"] = crp, ccol, cw
    hn2 = O.hec_heavy(crp, ccol, cw.astype(np.uint64), False, 100)
    vc2, nc2, _ = O.hec_map(hn2, 100)
    c2rp, c2col, c2w, _ = O.ref_build_coarse(crp, ccol, cw, vc2, nc2, 2)
    d["build2_vcmap"], d["build2_nc"] = vc2, np.array([nc2], np.uint32)
    d["build2_out_rp"], d["build2_out_col"], d["build2_out_w"] = c2rp, c2col, c2w
    # -- the reference's whole serial path on a 32x32 grid, 10 seeds (cuts)
    g3 = G.grid2d(32, 32)
    cuts = []
    for s in range(10):
        _, cut, _ = O.ref_partition_graph(g3.row_ptr, g3.col, rng_state=1000 + s, kind="serial", cutoff=50)
        cuts.append(cut)
    d["ref_grid32_cuts"] = np.array(cuts, np.uint64)
    np.savez_compressed(OUT, **d)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
