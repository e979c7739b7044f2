"""Python mirror of the sgpar.h partition API and of the explicit-context API.

The names, argument meanings and error behaviour follow cmg/sgpar.h
(sgp_load_graph :2262, sgp_load_config :2754, sgp_partition_graph :2363,
sgp_compute_partition :1969, sgp_use_partition :2666,
compute_partition_edit_distance :2343); all work runs in libsgpar_b200.so.
Host arrays are numpy; device arrays are CUDA torch tensors (their pointers are
passed through the C ABI, on the context's stream after a device sync).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib as L
from .graphs import CSR

_u32p = ctypes.POINTER(ctypes.c_uint32)
_dblp = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray, ct=ctypes.c_uint32):
    return a.ctypes.data_as(ctypes.POINTER(ct))


# ------------------------------------------------------------ sgpar.h API --
@dataclass
class Config:
    """config_t (sgpar.h:186-193)."""
    coarsening_alg: int = 4
    refine_alg: int = 0
    local_search_alg: int = 0
    num_partitions: int = 2
    num_iter: int = 10
    tol: float = 1e-10

    def to_c(self) -> L.config_t:
        c = L.config_t()
        c.coarsening_alg, c.refine_alg, c.local_search_alg = self.coarsening_alg, self.refine_alg, self.local_search_alg
        c.num_partitions, c.num_iter, c.tol = self.num_partitions, self.num_iter, self.tol
        return c


def load_config(path: str) -> Config:
    """sgp_load_config: six whitespace-separated fields (sgpar.h:2754)."""
    c = L.config_t()
    L.check(L.lib().sgp_load_config(path.encode(), ctypes.byref(c)), "sgp_load_config")
    return Config(c.coarsening_alg, c.refine_alg, c.local_search_alg, c.num_partitions, c.num_iter, c.tol)


def load_graph(path: str) -> CSR:
    """sgp_load_graph: the reference's binary CSR file (sgpar.h:2262)."""
    g = L.sgp_graph_t()
    L.check(L.lib().sgp_load_graph(ctypes.byref(g), path.encode()), "sgp_load_graph")
    n = g.nvertices
    m = 2 * g.nedges
    rp = np.ctypeslib.as_array(g.source_offsets, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(g.destination_indices, shape=(max(m, 1),))[:m].copy()
    L.lib().sgp_free_graph(ctypes.byref(g))
    return CSR(rp, col, None, path)


class _CGraph:
    """Keeps numpy buffers alive behind an sgp_graph_t."""

    def __init__(self, g: CSR):
        self.rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
        self.col = np.ascontiguousarray(g.col, dtype=np.uint32)
        self.w = None if g.w is None else np.ascontiguousarray(g.w, dtype=np.uint32)
        s = L.sgp_graph_t()
        s.nvertices = g.n
        s.nedges = g.m_directed // 2
        s.source_offsets = _ptr(self.rp)
        s.destination_indices = _ptr(self.col)
        s.eweights = _ptr(self.w) if self.w is not None else None
        self.s = s


@dataclass
class PCG32:
    """sgp_pcg32_random_t (sgpar.h:82)."""
    state: int = 0x853C49E6748FEA9B
    inc: int = 1

    def next(self) -> int:
        r = L.sgp_pcg32_random_t(self.state, self.inc)
        v = L.lib().sgp_pcg32_random_r(ctypes.byref(r))
        self.state = r.state
        return v


def partition_graph(g: CSR, config: Config, perc_imbalance_allowed: int = 0,
                    rng: Optional[PCG32] = None) -> tuple[np.ndarray, int]:
    """sgp_partition_graph (sgpar.h:2363): returns (part, edge_cut) and
    advances rng."""
    rng = rng or PCG32()
    cg = _CGraph(g)
    part = np.zeros(g.n, dtype=np.uint32)
    cut = ctypes.c_uint32(0)
    r = L.sgp_pcg32_random_t(rng.state, rng.inc)
    cfg = config.to_c()
    L.check(L.lib().sgp_partition_graph(_ptr(part), ctypes.byref(cut), ctypes.byref(cfg), perc_imbalance_allowed,
                                        cg.s, ctypes.byref(r)), "sgp_partition_graph")
    rng.state = r.state
    return part, cut.value


def compute_partition(evec: np.ndarray, g: CSR, num_partitions: int = 2, perc_imbalance_allowed: int = 0,
                      local_search_alg: int = 0) -> tuple[np.ndarray, int]:
    """sgp_compute_partition (sgpar.h:1969) on the device."""
    cg = _CGraph(g)
    ev = np.ascontiguousarray(evec, dtype=np.float64)
    part = np.zeros(g.n, dtype=np.uint32)
    cut = ctypes.c_uint32(0)
    L.check(L.lib().sgp_compute_partition(_ptr(part), num_partitions, ctypes.byref(cut), perc_imbalance_allowed,
                                          local_search_alg, _ptr(ev, ctypes.c_double), cg.s),
            "sgp_compute_partition")
    return part, cut.value


def use_partition(part: np.ndarray, g: CSR) -> tuple[CSR, CSR]:
    """sgp_use_partition (sgpar.h:2666): the two induced sub-graphs."""
    cg = _CGraph(g)
    p = np.ascontiguousarray(part, dtype=np.uint32)
    g1, g2 = L.sgp_graph_t(), L.sgp_graph_t()
    L.check(L.lib().sgp_use_partition(_ptr(p), cg.s, ctypes.byref(g1), ctypes.byref(g2)), "sgp_use_partition")
    out = []
    for s in (g1, g2):
        n, m = s.nvertices, s.nedges
        rp = np.ctypeslib.as_array(s.source_offsets, shape=(n + 1,)).copy()
        col = np.ctypeslib.as_array(s.destination_indices, shape=(max(m, 1),))[:m].copy()
        L.lib().sgp_free_graph(ctypes.byref(s))
        out.append(CSR(rp, col))
    return out[0], out[1]


def write_metrics(path: str, result: "Result", edge_cut_4way: int = 0, partition_diff: int = 0,
                  first: bool = True, last: bool = True) -> None:
    """Append ``result`` to the JSON metrics file ``path`` in the layout of
    the reference's ExperimentLoggerUtil::log (ExperimentLoggerUtil.cpp:145-192)."""
    if result.raw is None:
        raise ValueError("result has no C record (it was not produced by Partitioner)")
    L.check(L.lib().sgp_b200_write_metrics(path.encode(), ctypes.byref(result.raw), edge_cut_4way, partition_diff,
                                            int(first), int(last)), "sgp_b200_write_metrics")


def compute_partition_edit_distance(p1: np.ndarray, p2: np.ndarray) -> int:
    a = np.ascontiguousarray(p1, dtype=np.uint32)
    b = np.ascontiguousarray(p2, dtype=np.uint32)
    d = ctypes.c_uint32(0)
    L.check(L.lib().compute_partition_edit_distance(_ptr(a), _ptr(b), a.shape[0], ctypes.byref(d)),
            "compute_partition_edit_distance")
    return d.value


# ---------------------------------------------------- explicit context API --
@dataclass
class Result:
    part: object
    edgecut: int
    part0_size: int
    lam: float
    residual: float
    levels: int
    level_n: list = field(default_factory=list)
    level_m: list = field(default_factory=list)
    level_iters: list = field(default_factory=list)
    level_hec_rounds: list = field(default_factory=list)
    level_pi_ms: list = field(default_factory=list)
    iter_max_reached: bool = False
    rng_state: int = 0
    ms_total: float = 0.0
    ms_h2d: float = 0.0
    ms_coarsen: float = 0.0
    ms_eigen: float = 0.0
    ms_split: float = 0.0
    ms_d2h: float = 0.0
    kernel_launches: int = 0
    ms_map: float = 0.0
    ms_build: float = 0.0
    ls_swaps: int = 0           # local-search move pairs
    fm_passes: int = 0          # FM passes run
    fm_moves: int = 0           # FM moves applied
    raw: object = None          # the C result struct (for write_metrics)


class _DevArray:
    """__cuda_array_interface__ view of a device pointer (zero copy)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


class _GraphOwner:
    """Frees a library-allocated graph (sgp_b200_graph_free) when the last
    view of it goes away."""

    def __init__(self, g: L.sgp_b200_graph_t):
        self.g = g

    def __del__(self):
        try:
            L.lib().sgp_b200_graph_free(ctypes.byref(self.g))
        except Exception:
            pass


class _OwnedDevArray:
    """__cuda_array_interface__ view (int32) that keeps its owner alive."""

    def __init__(self, ptr: int, n: int, owner: _GraphOwner):
        self.owner = owner
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}


def _dptr(t) -> Optional[int]:
    return None if t is None else int(t.data_ptr())


def csr_write(path: str, g: CSR, id_bytes: int = 4) -> None:
    """The reference's binary CSR file (mtx2csr.cpp:266-289; id_bytes 8:
    mtx2csr_large.cpp) of a host graph."""
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(g.col, dtype=np.uint32)
    dg = L.sgp_b200_graph_t()
    dg.n, dg.m, dg.row_ptr, dg.col, dg.mem = g.n, len(col), rp.ctypes.data, col.ctypes.data, L.HOST
    L.check(L.lib().sgp_b200_csr_write(str(path).encode(), ctypes.byref(dg), id_bytes), "sgp_b200_csr_write")


def _mtx_info(i: L.sgp_b200_mtx_info_t) -> dict:
    return {name: getattr(i, name) for name, _ in L.sgp_b200_mtx_info_t._fields_}


class Partitioner:
    """One context (device, stream, memory pool) of libsgpar_b200."""

    def __init__(self, device: int = 0):
        self.device = device
        self._ctx = L.lib().sgp_b200_create(device)
        if not self._ctx:
            raise RuntimeError(f"sgp_b200_create({device}) failed: {L.last_error()}")

    def close(self) -> None:
        if self._ctx:
            L.lib().sgp_b200_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _sync():
        import torch
        torch.cuda.synchronize()

    # -- whole path
    def _graph(self, g, keep: list) -> L.sgp_b200_graph_t:
        dg = L.sgp_b200_graph_t()
        if isinstance(g, CSR):
            rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
            col = np.ascontiguousarray(g.col, dtype=np.uint32)
            keep += [rp, col]
            dg.n, dg.m = g.n, g.m_directed
            dg.row_ptr, dg.col = rp.ctypes.data, col.ctypes.data
            if g.w is not None:
                w = np.ascontiguousarray(g.w, dtype=np.uint32)
                keep.append(w)
                dg.w = w.ctypes.data
            dg.mem = L.HOST
        else:
            dg.n = int(g["row_ptr"].numel() - 1)
            dg.m = int(g["col"].numel())
            dg.row_ptr, dg.col = _dptr(g["row_ptr"]), _dptr(g["col"])
            dg.w = _dptr(g.get("w"))
            dg.mem = L.DEVICE
            self._sync()
        return dg

    @staticmethod
    def _options(cutoff, tol, mixed, rng_state, rng_inc, iter_cap, perc_imbalance,
                 refine_alg: int = 0, coarsener: int = 0, local_search_alg: int = 0,
                 fm_passes: int = 0, cluster_max_log2: int = 0,
                 cluster_blocks: int = 0) -> L.sgp_b200_options_t:
        o = L.sgp_b200_options_t()
        L.lib().sgp_b200_default_options(ctypes.byref(o))
        o.cutoff, o.tol, o.mixed, o.perc_imbalance = cutoff, tol, int(mixed), perc_imbalance
        o.iter_cap, o.rng_state, o.rng_inc = iter_cap, rng_state, rng_inc
        o.refine_alg = refine_alg
        o.coarsener = coarsener
        o.local_search_alg = local_search_alg
        o.fm_passes = fm_passes
        o.cluster_max_log2 = cluster_max_log2
        o.cluster_blocks = cluster_blocks
        return o

    @staticmethod
    def _part_target(n: int, part_out, o: L.sgp_b200_options_t):
        """(array, pointer) for a partition vector; sets o.part_mem."""
        if part_out is None:
            part_out = np.zeros(n, dtype=np.uint32)
        if isinstance(part_out, np.ndarray):
            o.part_mem = L.HOST
            return part_out, part_out.ctypes.data
        o.part_mem = L.DEVICE
        return part_out, _dptr(part_out)

    @staticmethod
    def _result(res: L.sgp_b200_result_t, part_out) -> Result:
        nl = res.levels
        return Result(part_out, res.edgecut, res.part0_size, res.lambda_, res.residual, nl,
                      list(res.level_n[:nl]), list(res.level_m[:nl]), list(res.level_iters[:nl]),
                      list(res.level_hec_rounds[:nl]), list(res.level_pi_ms[:nl]), bool(res.iter_max_reached),
                      res.rng_state,
                      res.ms_total, res.ms_h2d, res.ms_coarsen, res.ms_eigen, res.ms_split, res.ms_d2h,
                      res.kernel_launches, res.ms_map, res.ms_build, res.ls_swaps, res.fm_passes_run, res.fm_moves,
                      res)

    def partition(self, g, cutoff: int = 50, tol: float = 1e-10, mixed: bool = False,
                  rng_state: int = 0x853C49E6748FEA9B, rng_inc: int = 1, iter_cap: int = 0,
                  perc_imbalance: int = 0, part_out=None, refine_alg: int = 0, coarsener: int = 0,
                  local_search_alg: int = 0, fm_passes: int = 0, cluster_max_log2: int = 0,
                  cluster_blocks: int = 0) -> Result:
        """Partition ``g``: a host :class:`CSR` (numpy) or a dict of CUDA torch
        tensors ``{"row_ptr", "col", "w"}`` (device-resident input).  The
        partition is written to ``part_out`` (numpy or CUDA tensor) when
        given, else returned as numpy.  ``coarsener``: ``_lib.COARSEN_*``."""
        keep = []
        dg = self._graph(g, keep)
        o = self._options(cutoff, tol, mixed, rng_state, rng_inc, iter_cap, perc_imbalance, refine_alg, coarsener,
                          local_search_alg, fm_passes, cluster_max_log2, cluster_blocks)
        res = L.sgp_b200_result_t()
        part_out, res.part = self._part_target(dg.n, part_out, o)
        L.check(L.lib().sgp_b200_partition(self._ctx, ctypes.byref(dg), ctypes.byref(o), ctypes.byref(res)),
                "sgp_b200_partition")
        return self._result(res, part_out)

    def partition_4way(self, g, cutoff: int = 50, tol: float = 1e-10, mixed: bool = False,
                       rng_state: int = 0x853C49E6748FEA9B, rng_inc: int = 1, iter_cap: int = 0,
                       part_out=None, coarsener: int = 0) -> tuple:
        """The reference driver's 4-way mode (sgpar.cpp:62-89): returns
        (part4, cut of the bisection, cut4, rng state after the call) with
        part4[i] = 2 * bisection part + part inside its induced subgraph."""
        keep = []
        dg = self._graph(g, keep)
        o = self._options(cutoff, tol, mixed, rng_state, rng_inc, iter_cap, 0, 0, coarsener)
        part_out, ptr = self._part_target(dg.n, part_out, o)
        out = (L.c_u64 * 3)()
        L.check(L.lib().sgp_b200_partition_4way(self._ctx, ctypes.byref(dg), ctypes.byref(o), ptr, out),
                "sgp_b200_partition_4way")
        return part_out, int(out[0]), int(out[1]), int(out[2])

    def partition_batch(self, graphs: list, workers: int = 4, cutoff: int = 50, tol: float = 1e-10,
                        mixed: bool = False, rng_state: int = 0x853C49E6748FEA9B, rng_inc: int = 1,
                        iter_cap: int = 0, coarsener: int = 0, cluster_max_log2: int = 0,
                        cluster_blocks: int = 0) -> list:
        """Partition independent host graphs: ``workers`` host threads on
        separate streams coarsen them (largest first), one launch iterates the
        small coarse levels of every hierarchy (a block per hierarchy at a
        time), a second their mid-size levels (a cluster of blocks per
        hierarchy at a time; by default every level up to 2^23 cost units),
        and the workers finish the larger levels and the splits.  One
        :class:`Result` per graph, identical to partitioning it alone with the
        same options and the same ``cluster_max_log2`` and ``cluster_blocks``
        (23 and 2 by default here)."""
        keep = []
        cnt = max(1, len(graphs))
        arr = (L.sgp_b200_graph_t * cnt)()
        for i, g in enumerate(graphs):
            arr[i] = self._graph(g, keep)
        o = self._options(cutoff, tol, mixed, rng_state, rng_inc, iter_cap, 0, 0, coarsener,
                          cluster_max_log2=cluster_max_log2, cluster_blocks=cluster_blocks)
        o.part_mem = L.HOST
        res = (L.sgp_b200_result_t * cnt)()
        parts = []
        for i in range(len(graphs)):
            p = np.zeros(arr[i].n, dtype=np.uint32)
            parts.append(p)
            res[i].part = p.ctypes.data
        L.check(L.lib().sgp_b200_partition_batch(self._ctx, arr, len(graphs), ctypes.byref(o), res, workers),
                "sgp_b200_partition_batch")
        return [self._result(res[i], parts[i]) for i in range(len(graphs))]

    def last_timing(self) -> dict:
        """Phase times (ms) of the last call on this partitioner: CUDA-event
        phases of a partition, or the host wall times of a batch's phases
        (coarsen, the shared small-level launch as ``eigen``, the rest as
        ``split``)."""
        t = [ctypes.c_float(0) for _ in range(4)]
        L.check(L.lib().sgp_b200_last_timing(self._ctx, *[ctypes.byref(x) for x in t]), "sgp_b200_last_timing")
        return dict(zip(("total", "coarsen", "eigen", "split"), (x.value for x in t)))

    # -- per-kernel entry points (CUDA torch tensors)
    def fm_refine(self, row_ptr, col, part, max_passes: int = 16):
        """FM passes on a device bisection ``part`` (CUDA int32 tensor, updated
        in place): returns (cut, passes, moves)."""
        n = row_ptr.numel() - 1
        cut, passes, moves = ctypes.c_uint64(0), ctypes.c_uint32(0), ctypes.c_uint64(0)
        self._sync()
        L.check(L.lib().sgp_b200_fm_refine(self._ctx, n, _dptr(row_ptr), _dptr(col), _dptr(part), max_passes,
                                           ctypes.byref(cut), ctypes.byref(passes), ctypes.byref(moves)),
                "sgp_b200_fm_refine")
        return cut.value, passes.value, moves.value

    def coarsen_map(self, row_ptr, col, w=None, coarsener: int = 1, random_level: bool = False, seed: int = 1):
        """One level's mapping by an alternative coarsener (MATCH / MIS2 /
        GOSH): returns (vcmap CUDA tensor, nc, rounds)."""
        import torch
        n = row_ptr.numel() - 1
        vc = torch.empty(n, dtype=torch.int32, device=row_ptr.device)
        nc = ctypes.c_uint32(0)
        rounds = ctypes.c_int(0)
        wb = 0 if w is None else w.element_size()
        self._sync()
        L.check(L.lib().sgp_b200_coarsen_map(self._ctx, n, _dptr(row_ptr), _dptr(col), _dptr(w), wb, coarsener,
                                             int(random_level), seed, _dptr(vc), ctypes.byref(nc),
                                             ctypes.byref(rounds)), "sgp_b200_coarsen_map")
        return vc, nc.value, rounds.value

    def hec(self, row_ptr, col, w=None, random_level: bool = False, seed: int = 1):
        """Returns (hn, vcmap, nc, rounds) as CUDA tensors / ints."""
        import torch
        n = row_ptr.numel() - 1
        hn = torch.empty(n, dtype=torch.int32, device=row_ptr.device)
        vc = torch.empty(n, dtype=torch.int32, device=row_ptr.device)
        nc = ctypes.c_uint32(0)
        rounds = ctypes.c_int(0)
        wb = 0 if w is None else w.element_size()
        self._sync()
        L.check(L.lib().sgp_b200_hec(self._ctx, n, _dptr(row_ptr), _dptr(col), _dptr(w), wb, int(random_level),
                                     seed, _dptr(hn), _dptr(vc), ctypes.byref(nc), ctypes.byref(rounds)),
                "sgp_b200_hec")
        return hn, vc, nc.value, rounds.value

    def build_coarse(self, row_ptr, col, w, vcmap, nc: int, out_wbytes: int = 4):
        """Returns (c_row_ptr, c_col, c_w) CUDA tensors (int32 / int32 / int32|int64)."""
        import torch
        n = row_ptr.numel() - 1
        m = col.numel()
        dev = row_ptr.device
        crp = torch.empty(nc + 1, dtype=torch.int32, device=dev)
        ccol = torch.empty(max(m, 1), dtype=torch.int32, device=dev)
        cw = torch.empty(max(m, 1), dtype=torch.int32 if out_wbytes == 4 else torch.int64, device=dev)
        mc = ctypes.c_uint64(0)
        wb = 0 if w is None else w.element_size()
        self._sync()
        L.check(L.lib().sgp_b200_build_coarse(self._ctx, n, _dptr(row_ptr), _dptr(col), _dptr(w), wb, _dptr(vcmap),
                                              nc, out_wbytes, _dptr(crp), _dptr(ccol), _dptr(cw),
                                              ctypes.byref(mc)), "sgp_b200_build_coarse")
        k = mc.value
        return crp, ccol[:k], cw[:k]

    def power_iter(self, row_ptr, col, w, x_in, vcmap=None, tol: float = 1e-10, iter_cap: int = 0,
                   mixed: bool = False, residual: bool = True):
        """Returns (x_out, niter, lambda, residual)."""
        import torch
        n = row_ptr.numel() - 1
        out = torch.empty(n, dtype=torch.float64, device=row_ptr.device)
        it = ctypes.c_uint64(0)
        lam = ctypes.c_double(0)
        res = ctypes.c_double(0)
        wb = 0 if w is None else w.element_size()
        self._sync()
        L.check(L.lib().sgp_b200_power_iter(self._ctx, n, _dptr(row_ptr), _dptr(col), _dptr(w), wb, _dptr(x_in),
                                            _dptr(vcmap), _dptr(out), tol, iter_cap, int(mixed), ctypes.byref(it),
                                            ctypes.byref(lam), ctypes.byref(res) if residual else None),
                "sgp_b200_power_iter")
        return out, it.value, lam.value, res.value

    def split(self, row_ptr, col, evec, perc_imbalance: int = 0):
        """Returns (part CUDA tensor, edgecut)."""
        import torch
        n = row_ptr.numel() - 1
        part = torch.empty(n, dtype=torch.int32, device=row_ptr.device)
        cut = ctypes.c_uint64(0)
        self._sync()
        L.check(L.lib().sgp_b200_split(self._ctx, n, _dptr(row_ptr), _dptr(col), _dptr(evec), perc_imbalance,
                                       _dptr(part), ctypes.byref(cut)), "sgp_b200_split")
        return part, cut.value

    # -- MatrixMarket input (cmg/mtx2csr.cpp)
    def mtx_read(self, source, device_out: bool = False):
        """MatrixMarket coordinate text -> (graph of its largest connected
        component, info dict), computed on the device.  ``source``: a file
        path, ``bytes``, a uint8 numpy array, or a uint8 torch tensor (host
        memory, pinned or not, or CUDA) holding the text.  Returns a host
        ``CSR``, or with ``device_out`` a pair of CUDA int32 tensors (row_ptr,
        col)."""
        out = L.sgp_b200_graph_t()
        info = L.sgp_b200_mtx_info_t()
        mem = L.DEVICE if device_out else L.HOST
        where = "sgp_b200_mtx_parse"
        if isinstance(source, (bytes, bytearray, memoryview, np.ndarray)):
            buf = source if isinstance(source, np.ndarray) else np.frombuffer(source, dtype=np.uint8)
            buf = np.ascontiguousarray(buf).view(np.uint8).reshape(-1)
            rc = L.lib().sgp_b200_mtx_parse(self._ctx, buf.ctypes.data if buf.size else None, buf.size, L.HOST,
                                           mem, ctypes.byref(out), ctypes.byref(info))
        elif hasattr(source, "data_ptr"):
            if source.is_cuda:
                self._sync()
            rc = L.lib().sgp_b200_mtx_parse(self._ctx, _dptr(source) if source.numel() else None, source.numel(),
                                           L.DEVICE if source.is_cuda else L.HOST, mem, ctypes.byref(out),
                                           ctypes.byref(info))
        else:
            rc = L.lib().sgp_b200_mtx_read(self._ctx, str(source).encode(), mem, ctypes.byref(out),
                                          ctypes.byref(info))
            where = "sgp_b200_mtx_read"
        L.check(rc, where)
        n, m = out.n, out.m
        if device_out:
            # zero copy: the tensors share the library's allocation, which is
            # released when both are gone
            import torch
            owner = _GraphOwner(out)
            rp = torch.as_tensor(_OwnedDevArray(out.row_ptr, n + 1, owner), device="cuda")
            col = torch.as_tensor(_OwnedDevArray(out.col, m, owner), device="cuda") if m else \
                torch.zeros(0, dtype=torch.int32, device="cuda")
            return (rp, col), _mtx_info(info)
        try:
            rp = np.ctypeslib.as_array(ctypes.cast(out.row_ptr, _u32p), shape=(n + 1,)).copy()
            col = np.ctypeslib.as_array(ctypes.cast(out.col, _u32p), shape=(m,)).copy() if m else \
                np.zeros(0, dtype=np.uint32)
        finally:
            L.lib().sgp_b200_graph_free(ctypes.byref(out))
        return CSR(rp, col), _mtx_info(info)

    def mtx2csr(self, mtx_path: str, csr_path: str, id_bytes: int = 4) -> dict:
        """The reference command ``mtx2csr <MM file> <binary CSR file>``
        (``id_bytes`` 8: ``mtx2csr_hg``).  Returns the info dict."""
        info = L.sgp_b200_mtx_info_t()
        L.check(L.lib().sgp_b200_mtx2csr(self._ctx, str(mtx_path).encode(), str(csr_path).encode(), id_bytes,
                                        ctypes.byref(info)), "sgp_b200_mtx2csr")
        return _mtx_info(info)

    # -- hierarchy (lower boundary)
    def generate_coarse_graphs(self, g: CSR, cutoff: int = 50, rng: Optional[PCG32] = None) -> "Hierarchy":
        rng = rng or PCG32()
        rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
        col = np.ascontiguousarray(g.col, dtype=np.uint32)
        dg = L.sgp_b200_graph_t()
        dg.n, dg.m, dg.row_ptr, dg.col, dg.mem = g.n, g.m_directed, rp.ctypes.data, col.ctypes.data, L.HOST
        w = None
        if g.w is not None:
            w = np.ascontiguousarray(g.w, dtype=np.uint32)
            dg.w = w.ctypes.data
        r = L.sgp_pcg32_random_t(rng.state, rng.inc)
        h = ctypes.c_void_p()
        L.check(L.lib().sgp_b200_generate_coarse_graphs(self._ctx, ctypes.byref(dg), cutoff, ctypes.byref(r),
                                                        ctypes.byref(h)), "sgp_b200_generate_coarse_graphs")
        rng.state = r.state
        return Hierarchy(self, h.value)


class Hierarchy:
    """Device hierarchy handle (sgp_b200_hierarchy_t)."""

    def __init__(self, owner: Partitioner, handle: int):
        self.owner = owner
        self.h = handle

    def __len__(self) -> int:
        return L.lib().sgp_b200_hierarchy_levels(self.h)

    def level(self, l: int) -> dict:
        """Copies of level l as CUDA torch tensors."""
        import torch
        n, m = ctypes.c_uint32(0), ctypes.c_uint64(0)
        rp, col, w, vc = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        wb = ctypes.c_int(0)
        L.check(L.lib().sgp_b200_hierarchy_level(self.h, l, ctypes.byref(n), ctypes.byref(m), ctypes.byref(rp),
                                                 ctypes.byref(col), ctypes.byref(w), ctypes.byref(wb),
                                                 ctypes.byref(vc)), "sgp_b200_hierarchy_level")

        def view(p, cnt, ts):
            if not p.value or cnt == 0:
                return None
            return torch.as_tensor(_DevArray(p.value, cnt, ts), device="cuda").clone()
        vw = ctypes.c_void_p()
        L.check(L.lib().sgp_b200_hierarchy_vertex_weights(self.h, l, ctypes.byref(vw)),
                "sgp_b200_hierarchy_vertex_weights")
        out = {"n": n.value, "m": m.value, "row_ptr": view(rp, n.value + 1, "<u4"), "col": view(col, m.value, "<u4"),
               "wbytes": wb.value, "w": view(w, m.value, "<u4" if wb.value == 4 else "<u8"),
               "vcmap": view(vc, n.value, "<u4"), "vtx_w": view(vw, n.value, "<u4")}
        return out

    def eigensolve(self, rng: Optional[PCG32] = None, tol: float = 1e-10, mixed: bool = False,
                   iter_cap: int = 0) -> np.ndarray:
        rng = rng or PCG32()
        n0 = self.level(0)["n"]
        ev = np.zeros(n0, dtype=np.float64)
        r = L.sgp_pcg32_random_t(rng.state, rng.inc)
        L.check(L.lib().sgp_b200_eigensolve(self.owner._ctx, self.h, ctypes.byref(r), tol, int(mixed), iter_cap,
                                            ev.ctypes.data, L.HOST, None), "sgp_b200_eigensolve")
        rng.state = r.state
        return ev

    def free(self) -> None:
        if self.h:
            L.lib().sgp_b200_hierarchy_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
