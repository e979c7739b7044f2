"""The power iteration's autotuner (tune.cpp, eigen.cu autotune_level): the
first level of each shape on a device runs trial iterations of candidate
work splits and keeps the fastest in a per-device cache (memory and a text
file).  A tuned split changes only the order of floating-point sums, so the
partitions still match the oracle; a cached split is used without new trials;
SGPB_AUTOTUNE=0 keeps the built-in rules."""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def fresh_cache(tmp_path, monkeypatch):
    path = tmp_path / "pi_tune.txt"
    monkeypatch.setenv("SGPB_TUNE_CACHE", str(path))
    monkeypatch.setenv("SGPB_AUTOTUNE", "1")
    L.lib().sgp_b200_autotune_clear()
    yield path
    L.lib().sgp_b200_autotune_clear()


def read_cache(path):
    rows = []
    for line in path.read_text().splitlines():
        dev, shape, mode, div, units, ms_best, ms_rule = line.split()
        rows.append((dev, shape, int(mode), int(div), int(units), float(ms_best), float(ms_rule)))
    return rows


def check_against_oracle(g, r, seed):
    o = O.partition_graph(g.row_ptr, g.col, None, cutoff=50, tol=1e-10, rng_state=seed)
    assert r.level_n == o["level_n"] and r.rng_state == o["rng_state"]
    assert abs(r.lam - o["lambda"]) <= 1e-6 * abs(o["lambda"])
    assert abs(r.edgecut - o["edgecut"]) <= 0.02 * o["edgecut"] + 2
    assert r.edgecut == O.edge_cut(g.row_ptr, g.col, r.part)


def test_tuned_splits_cached_and_match_oracle(partitioner, fresh_cache):
    g = G.rmat(16, seed=4)
    r = partitioner.partition(g, rng_state=31)
    rows = read_cache(fresh_cache)
    assert rows, "no level was tuned"
    for dev, shape, mode, div, units, ms_best, ms_rule in rows:
        assert "B200" in dev or "SMs" in dev
        assert mode in (0, 5) and div > 0 and units in (8, 16, 32)
        assert 0 < ms_best <= ms_rule * (1 + 1e-9) or ms_rule == 0
    check_against_oracle(g, r, 31)
    # the same process again: cached splits, no new trials, identical bits
    r2 = partitioner.partition(g, rng_state=31)
    assert len(read_cache(fresh_cache)) == len(rows)
    assert np.array_equal(r2.part, r.part) and r2.lam == r.lam and r2.level_iters == r.level_iters


def test_splits_read_from_the_cache_file(partitioner, fresh_cache):
    """Splits written by another process (here: the file rewritten with a
    different split for every shape) are used as they are, without trials,
    and the partition still matches the oracle."""
    g = G.rmat(16, seed=4)
    partitioner.partition(g, rng_state=32)
    rows = read_cache(fresh_cache)
    forced = []
    for dev, shape, mode, div, units, a, b in rows:
        mode2 = 5 if mode == 0 else 0
        forced.append(f"{dev} {shape} {mode2} {64 if mode2 == 0 else 8} 32 {a:.6f} {b:.6f}")
    fresh_cache.write_text("\n".join(forced) + "\n")
    L.lib().sgp_b200_autotune_clear()
    r = partitioner.partition(g, rng_state=32)
    assert len(read_cache(fresh_cache)) == len(forced)   # nothing tuned again
    check_against_oracle(g, r, 32)


def test_autotune_off_uses_the_rules(partitioner, fresh_cache, monkeypatch):
    monkeypatch.setenv("SGPB_AUTOTUNE", "0")
    g = G.rmat(15, seed=6)
    r = partitioner.partition(g, rng_state=33)
    assert not fresh_cache.exists()
    check_against_oracle(g, r, 33)
