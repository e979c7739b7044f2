"""The reference's ``mtx2csr`` command (cmg/mtx2csr.cpp; ``--large`` for
cmg/mtx2csr_large.cpp's 64-bit layout) on the device:

    python -m ipdps_2021_graph_coarsening_b200.mtx2csr <MM file> <binary CSR file> [--large] [--device N]

Prints the same summary figures the reference prints (sizes before and after
dedupe, component count, largest component) and writes a byte-identical file.
"""
from __future__ import annotations

import argparse
import sys

from .api import Partitioner
from ._lib import SgparError


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="mtx2csr", description=__doc__.splitlines()[0])
    ap.add_argument("mtx")
    ap.add_argument("csr")
    ap.add_argument("--large", action="store_true", help="64-bit offsets and ids (mtx2csr_hg)")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    p = Partitioner(a.device)
    try:
        info = p.mtx2csr(a.mtx, a.csr, 8 if a.large else 4)
    except SgparError as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    finally:
        p.close()
    print(f"Matrix size: {info['rows']} {info['cols']} {info['entries_declared']}")
    print(f"{info['lines']} lines read from file.")
    print(f"After deduplication and self loop removal, n: {info['n_all']}, m: {info['m_all'] // 2}")
    if info["components"] == 1:
        print("There is just one connected component.")
    else:
        print(f"There are {info['components']} components and the largest component size is {info['n']}")
    print(f"Old edge count: {info['m_all'] // 2}, new edge count: {info['m'] // 2}")
    dev_ms = info["ms_parse"] + info["ms_rows"] + info["ms_components"] + info["ms_extract"]
    print(f"Converted in {info['ms_total']:.1f} ms (device phases {dev_ms:.1f} ms)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
