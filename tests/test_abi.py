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
