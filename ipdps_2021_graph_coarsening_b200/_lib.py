"""ctypes binding of ``libsgpar_b200.so`` (declarations: ``include/sgpar_b200.h``).

Loading fails loudly when the library is missing: there is no CPU fallback
for the partition path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsgpar_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "sgpar_b200.h")

c_u32, c_u64, c_int, c_dbl, c_flt = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double, ctypes.c_float
c_vp = ctypes.c_void_p
P = ctypes.POINTER

MAX_LEVELS = 202
OK, FAIL, ERR_INVALID, ERR_DEVICE, ERR_TOO_LARGE, ERR_BUDGET = 0, 1, 2, 3, 4, 5
HOST, DEVICE = 0, 1
COARSEN_HEC, COARSEN_MATCH, COARSEN_MIS2, COARSEN_GOSH, COARSEN_HEC_V3, COARSEN_GOSH_V2 = 0, 1, 2, 3, 4, 5
COARSEN_NONE, COARSEN_RATIO_STOP = 16, 32


class sgp_pcg32_random_t(ctypes.Structure):
    _fields_ = [("state", c_u64), ("inc", c_u64)]


class sgp_graph_t(ctypes.Structure):
    _fields_ = [("nvertices", c_u32), ("nedges", c_u32), ("source_offsets", P(c_u32)),
                ("edges_per_source", P(c_u32)), ("destination_indices", P(c_u32)),
                ("weighted_degree", P(c_u32)), ("eweights", P(c_u32))]


class config_t(ctypes.Structure):
    _fields_ = [("coarsening_alg", c_int), ("refine_alg", c_int), ("local_search_alg", c_int),
                ("num_iter", c_int), ("tol", c_dbl), ("num_partitions", c_int)]


class sgp_b200_graph_t(ctypes.Structure):
    _fields_ = [("n", c_u32), ("m", c_u64), ("row_ptr", c_vp), ("col", c_vp), ("w", c_vp), ("mem", c_int)]


class sgp_b200_options_t(ctypes.Structure):
    _fields_ = [("cutoff", c_u32), ("tol", c_dbl), ("mixed", c_int), ("perc_imbalance", c_int),
                ("iter_cap", c_u64), ("rng_state", c_u64), ("rng_inc", c_u64), ("part_mem", c_int),
                ("refine_alg", c_int), ("local_search_alg", c_int), ("fm_passes", c_u32), ("coarsener", c_int),
                ("cluster_max_log2", c_u32),
                ("cluster_blocks", c_u32)]


class sgp_b200_result_t(ctypes.Structure):
    _fields_ = [("part", c_vp), ("edgecut", c_u64), ("part0_size", c_u32), ("lambda_", c_dbl),
                ("residual", c_dbl), ("levels", c_int), ("level_n", c_u32 * MAX_LEVELS),
                ("level_m", c_u64 * MAX_LEVELS), ("level_iters", c_u64 * MAX_LEVELS),
                ("level_hec_rounds", c_int * MAX_LEVELS), ("level_pi_ms", c_flt * MAX_LEVELS),
                ("iter_max_reached", c_int),
                ("rng_state", c_u64), ("ms_total", c_flt), ("ms_h2d", c_flt), ("ms_coarsen", c_flt),
                ("ms_eigen", c_flt), ("ms_split", c_flt), ("ms_d2h", c_flt), ("kernel_launches", c_u32),
                ("ms_map", c_flt), ("ms_build", c_flt), ("ls_swaps", c_u32), ("fm_passes_run", c_u32),
                ("fm_moves", c_u64)]


class sgp_b200_mtx_info_t(ctypes.Structure):
    _fields_ = [("rows", c_u64), ("cols", c_u64), ("entries_declared", c_u64), ("lines", c_u64),
                ("bipartite", c_int), ("n_all", c_u32), ("m_all", c_u64), ("components", c_u32), ("n", c_u32),
                ("m", c_u64), ("ms_total", c_flt), ("ms_read", c_flt), ("ms_parse", c_flt), ("ms_rows", c_flt),
                ("ms_components", c_flt), ("ms_extract", c_flt), ("ms_out", c_flt),
                ("kernel_launches", c_u32)]


_SIGS = {
    # part 1: sgpar.h API
    "sgp_pcg32_random_r": (c_u32, [P(sgp_pcg32_random_t)]),
    "change_tol": (c_int, [c_dbl]),
    "sgp_load_graph": (c_int, [P(sgp_graph_t), ctypes.c_char_p]),
    "sgp_free_graph": (c_int, [P(sgp_graph_t)]),
    "sgp_load_partition": (c_int, [P(c_u32), c_u32, ctypes.c_char_p]),
    "sgp_load_config": (c_int, [ctypes.c_char_p, P(config_t)]),
    "compute_partition_edit_distance": (c_int, [P(c_u32), P(c_u32), c_u32, P(c_u32)]),
    "sgp_partition_graph": (c_int, [P(c_u32), P(c_u32), P(config_t), c_int, sgp_graph_t,
                                    P(sgp_pcg32_random_t)]),
    "sgp_compute_partition": (c_int, [P(c_u32), c_u32, P(c_u32), c_int, c_int, P(c_dbl), sgp_graph_t]),
    "sgp_use_partition": (c_int, [P(c_u32), sgp_graph_t, P(sgp_graph_t), P(sgp_graph_t)]),
    # part 2: explicit context
    "sgp_b200_create": (c_vp, [c_int]),
    "sgp_b200_destroy": (None, [c_vp]),
    "sgp_b200_last_error": (ctypes.c_char_p, []),
    "sgp_b200_stream": (c_vp, [c_vp]),
    "sgp_b200_default_options": (None, [P(sgp_b200_options_t)]),
    "sgp_b200_config_options": (c_int, [P(config_t), c_int, P(sgp_pcg32_random_t), P(sgp_b200_options_t)]),
    "sgp_b200_partition": (c_int, [c_vp, P(sgp_b200_graph_t), P(sgp_b200_options_t), P(sgp_b200_result_t)]),
    "sgp_b200_partition_4way": (c_int, [c_vp, P(sgp_b200_graph_t), P(sgp_b200_options_t), c_vp, P(c_u64)]),
    "sgp_b200_partition_batch": (c_int, [c_vp, P(sgp_b200_graph_t), c_int, P(sgp_b200_options_t),
                                         P(sgp_b200_result_t), c_int]),
    "sgp_b200_generate_coarse_graphs": (c_int, [c_vp, P(sgp_b200_graph_t), c_u32, P(sgp_pcg32_random_t),
                                                P(c_vp)]),
    "sgp_b200_hierarchy_levels": (c_int, [c_vp]),
    "sgp_b200_hierarchy_level": (c_int, [c_vp, c_int, P(c_u32), P(c_u64), P(c_vp), P(c_vp), P(c_vp),
                                         P(c_int), P(c_vp)]),
    "sgp_b200_hierarchy_vertex_weights": (c_int, [c_vp, c_int, P(c_vp)]),
    "sgp_b200_eigensolve": (c_int, [c_vp, c_vp, P(sgp_pcg32_random_t), c_dbl, c_int, c_u64, c_vp, c_int,
                                    P(sgp_b200_result_t)]),
    "sgp_b200_hierarchy_free": (None, [c_vp]),
    "sgp_b200_hec": (c_int, [c_vp, c_u32, c_vp, c_vp, c_vp, c_int, c_int, c_u64, c_vp, c_vp, P(c_u32),
                             P(c_int)]),
    "sgp_b200_build_coarse": (c_int, [c_vp, c_u32, c_vp, c_vp, c_vp, c_int, c_vp, c_u32, c_int, c_vp, c_vp,
                                      c_vp, P(c_u64)]),
    "sgp_b200_power_iter": (c_int, [c_vp, c_u32, c_vp, c_vp, c_vp, c_int, c_vp, c_vp, c_vp, c_dbl, c_u64,
                                    c_int, P(c_u64), P(c_dbl), P(c_dbl)]),
    "sgp_b200_split": (c_int, [c_vp, c_u32, c_vp, c_vp, c_vp, c_int, c_vp, P(c_u64)]),
    "sgp_b200_fm_refine": (c_int, [c_vp, c_u32, c_vp, c_vp, c_vp, c_u32, P(c_u64), P(c_u32), P(c_u64)]),
    "sgp_b200_coarsen_map": (c_int, [c_vp, c_u32, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_u64, c_vp, P(c_u32),
                                     P(c_int)]),
    "sgp_b200_autotune_clear": (None, []),
    "sgp_b200_last_timing": (c_int, [c_vp, P(c_flt), P(c_flt), P(c_flt), P(c_flt)]),
    "sgp_b200_write_metrics": (c_int, [ctypes.c_char_p, P(sgp_b200_result_t), c_u64, c_u64, c_int, c_int]),
    "sgp_b200_split_noalloc": (c_int, [c_vp, c_u32, c_vp, c_vp, c_vp, c_vp, c_vp]),
    # part 3: MatrixMarket input
    "sgp_b200_mtx_read": (c_int, [c_vp, ctypes.c_char_p, c_int, P(sgp_b200_graph_t), P(sgp_b200_mtx_info_t)]),
    "sgp_b200_mtx_parse": (c_int, [c_vp, c_vp, c_u64, c_int, c_int, P(sgp_b200_graph_t),
                                   P(sgp_b200_mtx_info_t)]),
    "sgp_b200_graph_free": (None, [P(sgp_b200_graph_t)]),
    "sgp_b200_csr_write": (c_int, [ctypes.c_char_p, P(sgp_b200_graph_t), c_int]),
    "sgp_b200_mtx2csr": (c_int, [c_vp, ctypes.c_char_p, ctypes.c_char_p, c_int, P(sgp_b200_mtx_info_t)]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load the library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run `python -m ipdps_2021_graph_coarsening_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_names() -> list[str]:
    return list(_SIGS)


def last_error() -> str:
    s = lib().sgp_b200_last_error()
    return s.decode() if s else ""


class SgparError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where} failed with code {code}: {last_error()}")
        self.code = code


def check(code: int, where: str) -> None:
    if code != 0:
        raise SgparError(code, where)
