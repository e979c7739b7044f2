"""Generate tests/golden/driver_metrics_{base,fourpart}.json: the metrics
files the config-file driver command (ipdps_2021_graph_coarsening_b200/sgpar_b200,
the reference's cmg/sgpar.cpp main) writes for a 64 x 48 grid with the
reference's two shipped configurations (cmg/base_config.txt: ten bisections;
cmg/fourpart_config.txt: ten 4-way partitions), rng state 2021.

Needs a CUDA device (the driver has no CPU path):

    python tests/golden/make_driver_metrics.py [output directory]

The files let the reference's experiment runner (cmg/jsonExperimentRunner.py
analyzeMetrics) be checked against real driver output where no GPU is.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ipdps_2021_graph_coarsening_b200 import graphs as G  # noqa: E402

DRIVER = os.path.join(ROOT, "ipdps_2021_graph_coarsening_b200", "sgpar_b200")
# the six fields of cmg/base_config.txt / cmg/fourpart_config.txt and their trailing token
CONFIGS = {"base": "4\n0\n0\n2\n10\n1e-10\nnone", "fourpart": "4\n0\n0\n4\n10\n1e-10\nnone"}


def main(out_dir: str) -> None:
    os.makedirs(out_dir, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        csr = os.path.join(tmp, "grid64x48.csr")
        G.write_csr(csr, G.grid2d(64, 48))
        for name, text in CONFIGS.items():
            cfg = os.path.join(tmp, f"{name}_config.txt")
            with open(cfg, "w") as f:
                f.write(text)
            out = os.path.join(out_dir, f"driver_metrics_{name}.json")
            if os.path.exists(out):
                os.remove(out)   # the driver appends
            p = subprocess.run([DRIVER, csr, out, cfg], capture_output=True, text=True,
                               env=dict(os.environ, SGPB_RNG_STATE="2021"))
            print(p.stdout, p.stderr)
            if p.returncode != 0:
                raise SystemExit(p.returncode)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
