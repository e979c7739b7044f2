"""ctypes bindings for the CPU checker (TEST INFRASTRUCTURE ONLY).

``liboracle.so`` is this project's C restatement of the reference path
(``oracle/sgpar_oracle.c``); ``libsgpar_ref_*.so`` is the reference's own
serial/OpenMP path compiled from cmg/sgpar.h (``oracle/ref_harness.cpp``).
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this module; the shipped library never imports it.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
c_u32, c_u64, c_int, c_dbl = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
u64ref = ctypes.POINTER(ctypes.c_uint64)
u32ref = ctypes.POINTER(ctypes.c_uint32)


def build() -> None:
    """Compile the oracle and, when the reference sources are present (the
    Makefile's REFERENCE_ROOT / REF_CMG, passed through the environment), the
    reference harness, with oracle/Makefile."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "oracle", "ref"], check=True)


def reference_root() -> str:
    """The reference checkout oracle/Makefile compiles from: the environment's
    REFERENCE_ROOT, else the Makefile's default (the one place that names it)."""
    if os.environ.get("REFERENCE_ROOT"):
        return os.environ["REFERENCE_ROOT"]
    import re
    with open(os.path.join(HERE, "Makefile")) as f:
        m = re.search(r"^REFERENCE_ROOT\s*\?=\s*(\S+)", f.read(), flags=re.M)
    return m.group(1) if m else ""


_orc = None


def lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_pcg32.argtypes = [u64ref, c_u64]
        L.orc_pcg32.restype = c_u32
        L.orc_hash_prio_key.argtypes = [c_u64, c_u32]
        L.orc_hash_prio_key.restype = c_u64
        L.orc_hash_rand_draw.argtypes = [c_u64, c_u32]
        L.orc_hash_rand_draw.restype = c_u64
        L.orc_hash_tiebreak.argtypes = [c_u64, c_u32, c_u32]
        L.orc_hash_tiebreak.restype = c_u32
        L.orc_hec_heavy.argtypes = [c_u32, u32p, u32p, ctypes.c_void_p, c_int, c_u64, u32p]
        L.orc_hec_heavy.restype = None
        L.orc_hec_map.argtypes = [c_u32, u32p, c_u64, u32p, u32ref]
        L.orc_hec_map.restype = c_int
        L.orc_hec_check.argtypes = [c_u32, u32p, u32p, c_u32]
        L.orc_hec_check.restype = c_int
        L.orc_build_coarse.argtypes = [c_u32, u32p, u32p, ctypes.c_void_p, u32p, c_u32,
                                       ctypes.c_void_p, ctypes.c_void_p, u32p, u32p, u64p]
        L.orc_build_coarse.restype = c_u64
        L.orc_dedupe_row.argtypes = [c_u32, u32p, u64p]
        L.orc_dedupe_row.restype = c_u32
        L.orc_power_iter.argtypes = [c_u32, u32p, u32p, ctypes.c_void_p, f64p, c_dbl, c_u64,
                                     ctypes.POINTER(c_dbl)]
        L.orc_power_iter.restype = c_u64
        L.orc_power_iter_nl.argtypes = L.orc_power_iter.argtypes
        L.orc_power_iter_nl.restype = c_u64
        L.orc_compute_partition.argtypes = [c_u32, u32p, u32p, f64p, c_int, u32p, u64ref]
        L.orc_compute_partition.restype = c_int
        L.orc_edge_cut.argtypes = [c_u32, u32p, u32p, u32p]
        L.orc_edge_cut.restype = c_u64
        L.orc_use_partition.argtypes = [c_u32, u32p, u32p, u32p, u32ref, u32p, u32p, u32ref, u32p, u32p]
        L.orc_use_partition.restype = c_int
        L.orc_partition_graph.argtypes = [c_u32, u32p, u32p, ctypes.c_void_p, c_u32, c_dbl,
                                          u64ref, c_u64, c_int, c_int, c_int, c_int, u32p, u64ref, f64p, f64p]
        L.orc_compute_partition_ls.argtypes = [c_u32, u32p, u32p, f64p, c_int, u32p, u64ref, u32ref]
        L.orc_compute_partition_ls.restype = c_int
        L.orc_fm_refine.argtypes = [c_u32, u32p, u32p, ctypes.c_void_p, u32p, c_u32, u64ref, u64ref]
        L.orc_fm_refine.restype = c_u32
        L.orc_match_map.argtypes = [c_u32, u32p, u32p, ctypes.c_void_p, c_int, c_u64, u32p, u32ref, u32ref]
        L.orc_match_map.restype = c_int
        L.orc_hec_v3_map.argtypes = [c_u32, u32p, u32p, u32ref]
        L.orc_hec_v3_map.restype = c_int
        L.orc_gosh_v2_map.argtypes = [c_u32, u32p, u32p, ctypes.c_void_p, c_u64, u32p, u32ref]
        L.orc_gosh_v2_map.restype = c_int
        L.orc_set_map.argtypes = [c_u32, u32p, u32p, c_int, c_u64, u32p, u32ref, u32ref]
        L.orc_set_map.restype = c_int
        L.orc_partition_graph.restype = c_int
        _orc = L
    return _orc


def _w64(w) -> tuple[Optional[np.ndarray], Optional[int]]:
    if w is None:
        return None, None
    w = np.ascontiguousarray(w, dtype=np.uint64)
    return w, w.ctypes.data


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


# ----------------------------------------------------------------- oracle --
def pcg32(state: int, inc: int, count: int) -> tuple[np.ndarray, int]:
    s = ctypes.c_uint64(state)
    out = np.array([lib().orc_pcg32(ctypes.byref(s), inc) for _ in range(count)], dtype=np.uint32)
    return out, s.value


def hec_heavy(row_ptr, col, w, random_level: bool, seed: int) -> np.ndarray:
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    hn = np.zeros(n, dtype=np.uint32)
    keep, wp = _w64(w)
    lib().orc_hec_heavy(n, rp, cl, wp, int(random_level), seed, hn)
    return hn


def hec_map(hn, seed: int) -> tuple[np.ndarray, int, int]:
    hn = _u32(hn)
    n = hn.shape[0]
    vc = np.zeros(n, dtype=np.uint32)
    nc = ctypes.c_uint32(0)
    rounds = lib().orc_hec_map(n, hn, seed, vc, ctypes.byref(nc))
    return vc, nc.value, rounds


def hec_check(hn, vcmap, nc: int) -> int:
    hn, vc = _u32(hn), _u32(vcmap)
    return lib().orc_hec_check(hn.shape[0], hn, vc, nc)


def build_coarse(row_ptr, col, w, vcmap, nc: int):
    """Returns (c_row_ptr, c_col, c_w uint64)."""
    rp, cl, vc = _u32(row_ptr), _u32(col), _u32(vcmap)
    n = rp.shape[0] - 1
    m = int(rp[-1])
    crp = np.zeros(nc + 1, dtype=np.uint32)
    ccol = np.zeros(m + 1, dtype=np.uint32)
    cw = np.zeros(m + 1, dtype=np.uint64)
    keep, wp = _w64(w)
    mc = lib().orc_build_coarse(n, rp, cl, wp, vc, nc, None, None, crp, ccol, cw)
    return crp, ccol[:mc].copy(), cw[:mc].copy()


def dedupe_row(dst, w):
    d = _u32(dst).copy()
    ww = np.ascontiguousarray(w, dtype=np.uint64).copy()
    m = lib().orc_dedupe_row(d.shape[0], d, ww)
    return d[:m], ww[:m]


def power_iter(row_ptr, col, w, u0, tol: float = 1e-10, iter_cap: int = 0):
    """Returns (u, niter, rayleigh quotient)."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    u = np.ascontiguousarray(u0, dtype=np.float64).copy()
    keep, wp = _w64(w)
    lam = ctypes.c_double(0)
    it = lib().orc_power_iter(n, rp, cl, wp, u, tol, iter_cap, ctypes.byref(lam))
    return u, int(it), lam.value


def power_iter_normalized(row_ptr, col, w, u0, tol: float = 1e-10, iter_cap: int = 0):
    """refine_alg 1 (normalized Laplacian).  Returns (u, niter, eigenvalue of
    the random-walk Laplacian)."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    u = np.ascontiguousarray(u0, dtype=np.float64).copy()
    keep, wp = _w64(w)
    lam = ctypes.c_double(0)
    it = lib().orc_power_iter_nl(n, rp, cl, wp, u, tol, iter_cap, ctypes.byref(lam))
    return u, int(it), lam.value


def compute_partition(row_ptr, col, evec, perc_imbalance: int = 0):
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    part = np.zeros(n, dtype=np.uint32)
    ec = ctypes.c_uint64(0)
    lib().orc_compute_partition(n, rp, cl, np.ascontiguousarray(evec, dtype=np.float64),
                                perc_imbalance, part, ctypes.byref(ec))
    return part, ec.value


def compute_partition_ls(row_ptr, col, evec, local_search_alg: int = 1):
    """The split plus the reference's local search -> (part, edgecut, swaps)."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    part = np.zeros(n, dtype=np.uint32)
    ec = ctypes.c_uint64(0)
    sw = ctypes.c_uint32(0)
    lib().orc_compute_partition_ls(n, rp, cl, np.ascontiguousarray(evec, dtype=np.float64), local_search_alg,
                                   part, ctypes.byref(ec), ctypes.byref(sw))
    return part, ec.value, sw.value


def fm_refine(row_ptr, col, w, part, max_passes: int = 16):
    """FM passes on a partition -> (part, cut, passes, moves)."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    p = np.ascontiguousarray(part, dtype=np.uint32).copy()
    keep, wp = _w64(w)
    cut = ctypes.c_uint64(edge_cut(rp, cl, p) if w is None else 0)
    mv = ctypes.c_uint64(0)
    passes = lib().orc_fm_refine(n, rp, cl, wp, p, max_passes, ctypes.byref(cut), ctypes.byref(mv))
    return p, cut.value, int(passes), mv.value


def edge_cut(row_ptr, col, part) -> int:
    rp, cl = _u32(row_ptr), _u32(col)
    return int(lib().orc_edge_cut(rp.shape[0] - 1, rp, cl, _u32(part)))


def use_partition(row_ptr, col, part):
    rp, cl, pt = _u32(row_ptr), _u32(col), _u32(part)
    n = rp.shape[0] - 1
    m = int(rp[-1])
    rp1 = np.zeros(n + 1, np.uint32); rp2 = np.zeros(n + 1, np.uint32)
    c1 = np.zeros(m + 1, np.uint32); c2 = np.zeros(m + 1, np.uint32)
    n1 = ctypes.c_uint32(0); n2 = ctypes.c_uint32(0)
    lib().orc_use_partition(n, rp, cl, pt, ctypes.byref(n1), rp1, c1, ctypes.byref(n2), rp2, c2)
    a, b = n1.value, n2.value
    return (rp1[:a + 1].copy(), c1[:rp1[a]].copy()), (rp2[:b + 1].copy(), c2[:rp2[b]].copy())


def match_map(row_ptr, col, w, random_level: bool, seed: int):
    """MATCH coarsener mapping -> (vcmap, nc, rounds)."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    keep, wp = _w64(w)
    vc = np.zeros(max(n, 1), np.uint32)
    nc, rounds = ctypes.c_uint32(0), ctypes.c_uint32(0)
    lib().orc_match_map(n, rp, cl, wp, int(random_level), seed, vc, ctypes.byref(nc), ctypes.byref(rounds))
    return vc[:n], nc.value, rounds.value


def hec_v3_map(row_ptr, col, w, random_level: bool, seed: int):
    """HEC_V3 mapping (HEC heavy neighbours, pointer-jumping construction)
    -> (vcmap, nc)."""
    hn = hec_heavy(row_ptr, col, w, random_level, seed)
    n = hn.shape[0]
    vc = np.zeros(max(n, 1), np.uint32)
    nc = ctypes.c_uint32(0)
    lib().orc_hec_v3_map(n, _u32(hn), vc, ctypes.byref(nc))
    return vc[:n], nc.value


def gosh_v2_map(row_ptr, col, w, seed: int):
    """GOSH_V2 mapping -> (vcmap, nc)."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    keep, wp = _w64(w)
    vc = np.zeros(max(n, 1), np.uint32)
    nc = ctypes.c_uint32(0)
    lib().orc_gosh_v2_map(n, rp, cl, wp, seed, vc, ctypes.byref(nc))
    return vc[:n], nc.value


def set_map(row_ptr, col, gosh: bool, seed: int):
    """MIS-2 (gosh False) or GOSH coarsener mapping -> (vcmap, nc, iterations)."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    vc = np.zeros(max(n, 1), np.uint32)
    nc, its = ctypes.c_uint32(0), ctypes.c_uint32(0)
    if lib().orc_set_map(n, rp, cl, int(gosh), seed, vc, ctypes.byref(nc), ctypes.byref(its)):
        raise RuntimeError("oracle coarsener left a vertex outside every aggregate")
    return vc[:n], nc.value, its.value


def partition_graph(row_ptr, col, w=None, cutoff: int = 50, tol: float = 1e-10,
                    rng_state: int = 42, rng_inc: int = 1, perc_imbalance: int = 0, refine_alg: int = 0,
                    coarsener: int = 0, local_search_alg: int = 0):
    """Whole multilevel path.  Returns dict(part, edgecut, evec, levels,
    lambda, niter (finest), level_n, level_iters, rng_state)."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    part = np.zeros(n, np.uint32)
    ev = np.zeros(n, np.float64)
    stats = np.zeros(3 + 2 * 202, np.float64)
    s = ctypes.c_uint64(rng_state)
    ec = ctypes.c_uint64(0)
    keep, wp = _w64(w)
    if lib().orc_partition_graph(n, rp, cl, wp, cutoff, tol, ctypes.byref(s), rng_inc, perc_imbalance,
                                 int(refine_alg), int(coarsener), int(local_search_alg), part, ctypes.byref(ec), ev,
                                 stats):
        raise RuntimeError("oracle coarsener left a vertex outside every aggregate")
    nl = int(stats[0])
    return dict(part=part, edgecut=ec.value, evec=ev, levels=nl, **{"lambda": stats[1]},
                niter=int(stats[2]), level_n=[int(stats[3 + 2 * l]) for l in range(nl)],
                level_iters=[int(stats[4 + 2 * l]) for l in range(nl)], rng_state=s.value)


# -------------------------------------------------------------- reference --
_refs: dict = {}


def ref_available(kind: str = "serial", cutoff: int = 50) -> bool:
    return os.path.exists(_ref_path(kind, cutoff))


def _ref_path(kind: str, cutoff: int) -> str:
    suffix = "" if cutoff == 50 else f"_c{cutoff}"
    return os.path.join(REF_DIR, f"libsgpar_ref_{kind}{suffix}.so")


def ref(kind: str = "serial", cutoff: int = 50):
    """The reference's own path: kind 'serial' (deterministic) or 'omp'."""
    key = (kind, cutoff)
    if key not in _refs:
        path = _ref_path(kind, cutoff)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.ref_power_iter.argtypes = [c_u32, u32p, u32p, vp, c_int, f64p, c_dbl, c_int]
        L.ref_power_iter_nl.argtypes = [c_u32, u32p, u32p, vp, f64p, c_dbl, c_int]
        L.ref_compute_partition.argtypes = [c_u32, u32p, u32p, f64p, c_int, u32p, u64ref, c_int]
        L.ref_compute_partition_ls.argtypes = [c_u32, u32p, u32p, f64p, c_int, c_int, u32p, u64ref, c_int]
        L.ref_build_coarse_msd.argtypes = [c_u32, u32p, u32p, vp, c_int, c_int, u32p, c_u32,
                                           u32p, u32p, u32p, u32p, u64ref]
        L.ref_coarsen_hec.argtypes = [c_u32, u32p, u32p, vp, c_int, u64ref, c_u64, u32p, u32ref]
        L.ref_partition_graph.argtypes = [c_u32, u32p, u32p, c_int, c_int, c_int, c_int, c_dbl, c_int,
                                          u64ref, c_u64, u32p, u64ref, c_int]
        L.ref_heap_deduplicate.argtypes = [u32p, u32p, u32p, u32p, u64ref]
        L.ref_hashmap_deduplicate.argtypes = [u32p, u32p, u32p, u32p, u64ref]
        _refs[key] = L
    return _refs[key]


def ref_power_iter(row_ptr, col, w, u0, final_level: bool, tol: float = 1e-10, kind: str = "serial"):
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    u = np.ascontiguousarray(u0, dtype=np.float64).copy()
    wk = None if w is None else _u32(w)
    ref(kind).ref_power_iter(n, rp, cl, None if wk is None else wk.ctypes.data, int(final_level),
                             u, tol, 1)
    return u


def ref_power_iter_normalized(row_ptr, col, w, u0, tol: float = 1e-10, kind: str = "serial"):
    """The reference's refine_alg 1 power iteration on a coarse level."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    u = np.ascontiguousarray(u0, dtype=np.float64).copy()
    wk = None if w is None else _u32(w)
    ref(kind).ref_power_iter_nl(n, rp, cl, None if wk is None else wk.ctypes.data, u, tol, 1)
    return u


def ref_compute_partition(row_ptr, col, evec, perc_imbalance: int = 0, kind: str = "serial"):
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    part = np.zeros(n, np.uint32)
    ec = ctypes.c_uint64(0)
    ref(kind).ref_compute_partition(n, rp, cl, np.ascontiguousarray(evec, dtype=np.float64).copy(),
                                    perc_imbalance, part, ctypes.byref(ec), 1)
    return part, ec.value


def ref_compute_partition_ls(row_ptr, col, evec, local_search_alg: int = 1, kind: str = "serial"):
    """The reference's sgp_compute_partition with its local search."""
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    part = np.zeros(n, np.uint32)
    ec = ctypes.c_uint64(0)
    ref(kind).ref_compute_partition_ls(n, rp, cl, np.ascontiguousarray(evec, dtype=np.float64).copy(), 0,
                                       local_search_alg, part, ctypes.byref(ec), 1)
    return part, ec.value


def ref_build_coarse(row_ptr, col, w, vcmap, nc: int, level: int, coarsening_alg: int = 4,
                     kind: str = "serial"):
    """The reference's coarse build on a given mapping, canonicalised to
    compact CSR with rows sorted by destination.  Returns (rp, col, w, nedges)."""
    rp, cl, vc = _u32(row_ptr), _u32(col), _u32(vcmap).copy()
    n = rp.shape[0] - 1
    m = int(rp[-1])
    wk = None if w is None else _u32(w)
    off = np.zeros(nc + 1, np.uint32); cnt = np.zeros(nc, np.uint32)
    oc = np.zeros(m + 1, np.uint32); ow = np.zeros(m + 1, np.uint32)
    ne = ctypes.c_uint64(0)
    ref(kind).ref_build_coarse_msd(n, rp, cl, None if wk is None else wk.ctypes.data, level,
                                   coarsening_alg, vc, nc, off, cnt, oc, ow, ctypes.byref(ne))
    out_rp = np.zeros(nc + 1, np.uint32)
    out_rp[1:] = np.cumsum(cnt, dtype=np.uint64)
    cols, wts = [], []
    for c in range(nc):
        s = int(off[c])
        cc = oc[s:s + cnt[c]]; ww = ow[s:s + cnt[c]]
        o = np.argsort(cc, kind="stable")
        cols.append(cc[o]); wts.append(ww[o])
    ccol = np.concatenate(cols) if cols else np.zeros(0, np.uint32)
    cw = np.concatenate(wts) if wts else np.zeros(0, np.uint32)
    return out_rp, ccol, cw, ne.value


def ref_partition_graph(row_ptr, col, rng_state: int, rng_inc: int = 1, tol: float = 1e-10,
                        coarsening_alg: int = 4, num_partitions: int = 2, kind: str = "serial",
                        cutoff: int = 50, quiet: bool = True):
    rp, cl = _u32(row_ptr), _u32(col)
    n = rp.shape[0] - 1
    part = np.zeros(n, np.uint32)
    s = ctypes.c_uint64(rng_state)
    ec = ctypes.c_uint64(0)
    rc = ref(kind, cutoff).ref_partition_graph(n, rp, cl, coarsening_alg, 0, 0, num_partitions, tol, 0,
                                               ctypes.byref(s), rng_inc, part, ctypes.byref(ec),
                                               int(quiet))
    if rc != 0:
        raise RuntimeError(f"reference sgp_partition_graph returned {rc}")
    return part, ec.value, s.value
