"""Metrics files written by the config-file driver command on a B200
(tests/golden/driver_metrics_{base,fourpart}.json, made by
tests/golden/make_driver_metrics.py from a 64 x 48 grid with the reference's
base and four-part configurations) against the reference's own experiment
runner: cmg/jsonExperimentRunner.py's analyzeMetrics (:113-125) loads them
unchanged and produces its statistics.  The runner is read from the
reference checkout when it is present (REFERENCE_ROOT, as for
oracle/Makefile); the layout checks run everywhere.  No GPU needed."""
import importlib.util
import json
import os
import sys
import types

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = {k: os.path.join(HERE, "golden", f"driver_metrics_{k}.json") for k in ("base", "fourpart")}


@pytest.mark.parametrize("name", sorted(FILES))
def test_driver_metrics_layout(name):
    recs = json.load(open(FILES[name]))
    assert len(recs) == 10   # num_iter of both configurations
    for r in recs:
        assert r["edge-cut"] > 0 and r["number-coarse-levels"] == len(r["coarse-levels"])
        lv = r["coarse-levels"]
        assert [x["number-vertices"] for x in lv] == sorted(x["number-vertices"] for x in lv)
        assert lv[-1]["number-vertices"] == 64 * 48 and lv[-1]["unrefined-edge-cut"] == r["edge-cut"]
        if name == "fourpart":
            assert r["edge-cut-four-way"] > r["edge-cut"]
        else:
            assert r["edge-cut-four-way"] == 0


def reference_runner():
    from oracle import bindings as O
    path = os.path.join(O.reference_root(), "cmg", "jsonExperimentRunner.py")
    if not os.path.exists(path):
        pytest.skip("reference checkout not present")
    # the runner imports the third-party `parse` package for a log-reprocessing
    # helper that analyzeMetrics does not use; it is not installed here
    sys.modules.setdefault("parse", types.SimpleNamespace(parse=None))
    spec = importlib.util.spec_from_file_location("jsonExperimentRunner", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("name", sorted(FILES))
def test_reference_runner_aggregates_driver_metrics(name, tmp_path):
    mod = reference_runner()
    log = tmp_path / f"{name}_Sampling_Data.txt"
    mod.analyzeMetrics(FILES[name], str(log))
    stats = json.load(open(tmp_path / f"{name}_Sampling_Data.json"))
    cuts = [r["edge-cut"] for r in json.load(open(FILES[name]))]
    assert stats["edge-cut"]["min"] == min(cuts) and stats["edge-cut"]["max"] == max(cuts)
    assert "total-duration-seconds" in stats and "coarse-levels" in stats
    assert "edge-cut" in log.read_text()
