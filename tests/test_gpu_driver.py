"""The config-file driver command `sgpar_b200 <csr> <metrics.json> <config>
[best_partition]` (csrc/sgpar_main.c, the reference's cmg/sgpar.cpp:11-106)
run as a process on the GPU, with the two configurations the reference ships:

* base_config.txt (cmg/base_config.txt: coarsening_alg 4, refine_alg 0,
  local_search_alg 0, num_partitions 2, num_iter 10, tol 1e-10): ten
  bisections with one rng carried through them;
* fourpart_config.txt (cmg/fourpart_config.txt: the same with
  num_partitions 4): each bisection followed by the bisections of its two
  induced sub-graphs, the 4-way cut the sum of the three.

Every record of the metrics file must equal the library's own calls with the
same carried rng (the bisection through sgp_b200_partition, the 4-way cut
through sgp_b200_partition_4way), the printed minimum must be the smallest
record, and a best-partition file must give the edit distances of
compute_partition_edit_distance.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import graphs as G

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(os.path.dirname(HERE), "ipdps_2021_graph_coarsening_b200", "sgpar_b200")

# the six fields of cmg/base_config.txt and cmg/fourpart_config.txt, one per
# line, and their trailing token
BASE_CONFIG = "4\n0\n0\n2\n10\n1e-10\nnone"
FOURPART_CONFIG = "4\n0\n0\n4\n10\n1e-10\nnone"
SEED = 2021


def run_driver(tmp_path, g, config_text, best=None, name="metrics.json"):
    csr = tmp_path / "graph.csr"
    if not csr.exists():
        G.write_csr(str(csr), g)
    cfg = tmp_path / "config.txt"
    cfg.write_text(config_text)
    metrics = tmp_path / name
    args = [DRIVER, str(csr), str(metrics), str(cfg)] + ([str(best)] if best else [])
    env = dict(os.environ, SGPB_RNG_STATE=str(SEED))
    p = subprocess.run(args, capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    m = re.search(r"min edgecut found is (\d+)", p.stdout)
    assert m, p.stdout
    return json.load(open(metrics)), int(m.group(1)), p.stdout


def test_base_config_ten_bisections(tmp_path, partitioner):
    g = G.grid2d_holes(90, 70, 0.1, 2)
    recs, cut_min, out = run_driver(tmp_path, g, BASE_CONFIG)
    assert f"n: {g.n}, m: {g.m_undirected}" in out
    assert "coarsening_alg: 4, refine_alg: 0, local_alg 0, num_iter 10" in out
    assert len(recs) == 10
    state = SEED
    for rec in recs:
        r = partitioner.partition(g, rng_state=state)
        assert rec["edge-cut"] == r.edgecut
        assert rec["edge-cut-four-way"] == 0 and rec["partition-diff"] == 0
        assert rec["number-coarse-levels"] == r.levels
        assert [x["number-vertices"] for x in rec["coarse-levels"]] == r.level_n[::-1]
        assert [x["refine-iterations"] for x in rec["coarse-levels"]] == r.level_iters[::-1]
        state = r.rng_state
    assert cut_min == min(rec["edge-cut"] for rec in recs)
    # the rng is carried: the ten bisections are not all the same
    assert len({rec["edge-cut"] for rec in recs}) > 1 or len({tuple(x["refine-iterations"] for x in rec["coarse-levels"])
                                                          for rec in recs}) > 1


def test_fourpart_config(tmp_path, partitioner):
    g = G.rgg3d(20000, seed=5)
    recs, cut_min, _ = run_driver(tmp_path, g, FOURPART_CONFIG)
    assert len(recs) == 10
    state = SEED
    for rec in recs:
        _, cut2, cut4, state = partitioner.partition_4way(g, rng_state=state)
        assert rec["edge-cut"] == cut2 and rec["edge-cut-four-way"] == cut4
        assert cut4 >= cut2
    assert cut_min == min(rec["edge-cut"] for rec in recs)


def test_best_partition_edit_distance(tmp_path, partitioner):
    g = G.grid2d(60, 50)
    r = partitioner.partition(g, rng_state=SEED)
    best = tmp_path / "best.txt"
    best.write_text("\n".join(str(int(x)) for x in r.part) + "\n")
    one = BASE_CONFIG.replace("\n10\n", "\n3\n")   # num_iter 3
    recs, _, _ = run_driver(tmp_path, g, one, best=best)
    from ipdps_2021_graph_coarsening_b200.api import compute_partition_edit_distance
    state = SEED
    for k, rec in enumerate(recs):
        rk = partitioner.partition(g, rng_state=state)
        state = rk.rng_state
        assert rec["partition-diff"] == compute_partition_edit_distance(np.asarray(rk.part), np.asarray(r.part))
    assert recs[0]["partition-diff"] == 0


def test_driver_reports_errors(tmp_path):
    cfg = tmp_path / "c.txt"
    cfg.write_text(BASE_CONFIG)
    p = subprocess.run([DRIVER, str(tmp_path / "missing.csr"), str(tmp_path / "m.json"), str(cfg)],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 1 and "reading the graph" in p.stderr
