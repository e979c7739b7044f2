"""The C-ABI library loads, exports every entry point of include/sgpar_b200.h,
and its host-only entry points (file loaders, PCG32, edit distance) behave
like the reference's.  No kernel is launched here."""
import os
import re

import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import api, graphs as G
from oracle import bindings as O


def header_functions():
    txt = open(L.HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b([a-z_][a-z0-9_]*)\s*\(", txt, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "sizeof", "defined")))


def test_header_declares_the_sgpar_api():
    names = header_functions()
    for n in ("sgp_load_graph", "sgp_free_graph", "sgp_load_config", "sgp_load_partition",
              "compute_partition_edit_distance", "sgp_partition_graph", "sgp_compute_partition",
              "sgp_use_partition", "sgp_pcg32_random_r", "change_tol"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(header_functions()) <= set(L.exported_names())


def test_pcg32_matches_oracle():
    r = api.PCG32(state=42, inc=54)
    ours = [r.next() for _ in range(20)]
    ref, _ = O.pcg32(42, 54, 20)
    assert ours == ref.tolist()


def test_load_config(tmp_path):
    p = tmp_path / "base_config.txt"
    p.write_text("4\n0\n0\n2\n10\n1e-10\nnone")   # the reference's base_config.txt layout
    c = api.load_config(str(p))
    assert (c.coarsening_alg, c.refine_alg, c.local_search_alg, c.num_partitions, c.num_iter) == (4, 0, 0, 2, 10)
    assert c.tol == 1e-10
    bad = tmp_path / "bad.txt"
    bad.write_text("4 0")
    with pytest.raises(L.SgparError):
        api.load_config(str(bad))


def test_load_graph_roundtrip(tmp_path):
    g = G.rmat(8, seed=3)
    path = str(tmp_path / "g.csr")
    G.write_csr(path, g)
    h = api.load_graph(path)
    assert np.array_equal(h.row_ptr, g.row_ptr) and np.array_equal(h.col, g.col)
    with pytest.raises(L.SgparError):
        api.load_graph(str(tmp_path / "missing.csr"))


def test_edit_distance():
    a = np.array([0, 0, 1, 1, 0, 1], np.uint32)
    b = 1 - a
    assert api.compute_partition_edit_distance(a, a) == 0
    assert api.compute_partition_edit_distance(a, b) == 0   # label swap
    c = a.copy(); c[0] = 1; c[2] = 0
    assert api.compute_partition_edit_distance(a, c) == 1


def test_no_silent_cpu_path_without_a_device():
    """Without a CUDA device the context cannot be created: the partition path
    fails loudly instead of falling back to the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    assert not L.lib().sgp_b200_create(0)
    assert L.last_error()


# keys of one record of the reference's metrics file (ExperimentLoggerUtil.cpp:145-192)
METRIC_KEYS = ["edge-cut", "edge-cut-four-way", "partition-diff", "total-duration-seconds",
               "coarsen-duration-seconds", "refine-duration-seconds", "number-coarse-levels",
               "level-1-first-two-passes-assign-rate", "level-1-total-passes",
               "level-2-first-two-passes-assign-rate", "level-2-total-passes"] + \
    [f"{k}-duration-seconds" for k in ["coarsen-map", "coarsen-build", "coarsen-count", "coarsen-prefix-sum",
                                       "coarsen-bucket", "coarsen-dedupe", "coarsen-radix-sort",
                                       "coarsen-radix-dedupe", "coarsen-write-graph", "coarsen-permute",
                                       "coarsen-map-construct", "fm-refine", "fm-recoarsen", "heavy"]] + \
    ["coarse-levels"]
LEVEL_KEYS = ["refine-iterations", "iteration-max-reached", "number-vertices", "unrefined-edge-cut"]


def test_metrics_file_has_the_reference_layout(tmp_path):
    """Two records appended like the reference driver's loop (first / last
    flags) form one JSON list with the reference's keys, in its order."""
    import json
    from ipdps_2021_graph_coarsening_b200.api import Result, write_metrics
    recs = []
    for k in range(2):
        r = L.sgp_b200_result_t()
        r.edgecut, r.levels = 100 + k, 3
        for i, (n, it) in enumerate([(1000, 12), (300, 40), (40, 700)]):
            r.level_n[i], r.level_iters[i], r.level_hec_rounds[i] = n, it, 5 + i
        r.ms_h2d, r.ms_coarsen, r.ms_eigen, r.ms_split, r.ms_map, r.ms_build = 1.0, 4.0, 20.0, 2.0, 1.5, 2.5
        recs.append(Result(None, r.edgecut, 0, 0.0, 0.0, 3, raw=r))
    path = str(tmp_path / "metrics.json")
    write_metrics(path, recs[0], edge_cut_4way=250, first=True, last=False)
    write_metrics(path, recs[1], edge_cut_4way=260, first=False, last=True)
    data = json.load(open(path))
    assert len(data) == 2
    for k, d in enumerate(data):
        assert list(d) == METRIC_KEYS
        assert d["edge-cut"] == 100 + k and d["edge-cut-four-way"] == 250 + 10 * k
        assert abs(d["total-duration-seconds"] - 0.025) < 1e-12       # upload + coarsen + eigensolve
        assert abs(d["coarsen-duration-seconds"] - 0.005) < 1e-12
        assert abs(d["coarsen-map-duration-seconds"] - 0.0015) < 1e-12
        assert d["number-coarse-levels"] == 3 and d["level-1-total-passes"] == 5 and d["level-2-total-passes"] == 6
        lv = d["coarse-levels"]
        assert [list(x) for x in lv] == [LEVEL_KEYS] * 3
        assert [x["number-vertices"] for x in lv] == [40, 300, 1000]      # coarsest first
        assert [x["unrefined-edge-cut"] for x in lv] == [0, 0, 100 + k]  # the finest carries the cut
        assert [x["refine-iterations"] for x in lv] == [700, 40, 12]


def test_config_options_follow_sgp_partition_graph():
    """coarsening_alg's bits select the coarsener as sgpar.h:2457-2475 reads
    them; the tolerance, refine and local-search choices and the rng pass
    through; refine_alg outside {0, 1} is rejected."""
    import ctypes
    cases = [(4, L.COARSEN_HEC), (1, L.COARSEN_MATCH | L.COARSEN_RATIO_STOP), (5, L.COARSEN_MATCH | L.COARSEN_RATIO_STOP),
             (16, L.COARSEN_NONE), (17, L.COARSEN_NONE)]
    for alg, want in cases:
        c = L.config_t(coarsening_alg=alg, refine_alg=1, local_search_alg=1, num_iter=3, tol=1e-8,
                       num_partitions=2)
        rng = L.sgp_pcg32_random_t(state=77, inc=5)
        o = L.sgp_b200_options_t()
        assert L.lib().sgp_b200_config_options(ctypes.byref(c), 0, ctypes.byref(rng), ctypes.byref(o)) == L.OK
        assert o.coarsener == want and o.refine_alg == 1 and o.local_search_alg == 1 and o.tol == 1e-8
        assert o.rng_state == 77 and o.rng_inc == 5 and o.perc_imbalance == 0 and o.cutoff == 50
    c = L.config_t(coarsening_alg=4, refine_alg=2, local_search_alg=0, num_iter=1, tol=1e-10, num_partitions=2)
    rng = L.sgp_pcg32_random_t(state=1, inc=1)
    assert L.lib().sgp_b200_config_options(ctypes.byref(c), 0, ctypes.byref(rng),
                                           ctypes.byref(L.sgp_b200_options_t())) == L.ERR_INVALID


DRIVER = os.path.join(os.path.dirname(L.LIB_PATH), "sgpar_b200")


def test_driver_command_usage():
    """The config-file driver command is built and prints the reference's
    usage line, exiting EXIT_FAILURE, when arguments are missing."""
    import subprocess
    assert os.path.exists(DRIVER)
    p = subprocess.run([DRIVER, "only-one"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1
    assert "You input 2 args" in p.stdout
    assert "csr_filename metrics_filename config_file" in p.stderr
