"""Seeded synthetic graphs with the shapes of the benchmark configurations.

Thin ctypes wrapper over ``libsgpgen.so`` (``csrc/graphgen.cpp``).  Every graph
is a symmetric CSR with sorted rows, no self loops and no duplicate entries,
restricted to its largest connected component -- the input invariants the
reference's converter establishes (cmg/mtx2csr.cpp:132-264).

Graphs are returned as :class:`CSR` (numpy arrays, uint32).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


class _CSR(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("m", ctypes.c_uint64),
                ("row_ptr", ctypes.POINTER(ctypes.c_uint32)),
                ("col", ctypes.POINTER(ctypes.c_uint32)),
                ("w", ctypes.POINTER(ctypes.c_uint32))]


@dataclass
class CSR:
    """Symmetric CSR graph: ``row_ptr[n+1]``, ``col[m]``, optional ``w[m]``."""
    row_ptr: np.ndarray
    col: np.ndarray
    w: Optional[np.ndarray] = None
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.row_ptr.shape[0] - 1)

    @property
    def m_directed(self) -> int:
        return int(self.row_ptr[-1])

    @property
    def m_undirected(self) -> int:
        return self.m_directed // 2


_lib = None


def _gen():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "libsgpgen.so")
        if not os.path.exists(path):
            raise RuntimeError("libsgpgen.so is not built; run ipdps_2021_graph_coarsening_b200.build.build_all()")
        lib = ctypes.CDLL(path)
        P = ctypes.POINTER(_CSR)
        u32, u64, dbl, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_int
        lib.sgpgen_grid2d.argtypes = [u32, u32, P]
        lib.sgpgen_grid2d_holes.argtypes = [u32, u32, dbl, u64, P]
        lib.sgpgen_rmat.argtypes = [i32, i32, dbl, dbl, dbl, u64, i32, P]
        lib.sgpgen_er.argtypes = [u32, dbl, u64, P]
        lib.sgpgen_rgg3d.argtypes = [u32, dbl, u64, P]
        lib.sgpgen_chunglu.argtypes = [u32, dbl, dbl, dbl, u32, u64, P]
        lib.sgpgen_write_csr.argtypes = [ctypes.c_char_p, P]
        lib.sgpgen_free.argtypes = [P]
        lib.sgpgen_free.restype = None
        _lib = lib
    return _lib


def _take(raw: _CSR, name: str) -> CSR:
    n, m = raw.n, raw.m
    rp = np.ctypeslib.as_array(raw.row_ptr, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(raw.col, shape=(max(m, 1),))[:m].copy()
    w = None
    if bool(raw.w):
        w = np.ctypeslib.as_array(raw.w, shape=(max(m, 1),))[:m].copy()
    _gen().sgpgen_free(ctypes.byref(raw))
    return CSR(rp, col, w, name)


def _call(fn, *args, name: str) -> CSR:
    raw = _CSR()
    rc = fn(*args, ctypes.byref(raw))
    if rc != 0:
        raise RuntimeError(f"graph generator {name} failed (rc={rc})")
    return _take(raw, name)


def grid2d(nx: int, ny: int) -> CSR:
    """nx*ny 5-point grid, vertex (r, c) = r*nx + c."""
    return _call(_gen().sgpgen_grid2d, nx, ny, name=f"grid{nx}x{ny}")


def grid2d_holes(nx: int, ny: int, frac_removed: float = 0.1, seed: int = 1) -> CSR:
    return _call(_gen().sgpgen_grid2d_holes, nx, ny, frac_removed, seed, name=f"holes{nx}x{ny}")


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1, scramble: bool = True) -> CSR:
    """R-MAT, symmetrised, duplicates merged, self loops dropped, LCC kept."""
    return _call(_gen().sgpgen_rmat, scale, edge_factor, a, b, c, seed, int(scramble),
                 name=f"rmat{scale}")


def erdos_renyi(n: int, mean_degree: float = 8.0, seed: int = 1) -> CSR:
    return _call(_gen().sgpgen_er, n, mean_degree, seed, name=f"er{n}")


def rgg3d(n: int, mean_degree: float = 12.0, seed: int = 1, radius: Optional[float] = None) -> CSR:
    """3D random geometric graph in the unit cube; the radius defaults to the
    one whose interior expected degree is ``mean_degree`` (boundary cells lower
    the measured mean slightly)."""
    if radius is None:
        radius = (mean_degree / (n * 4.0 / 3.0 * math.pi)) ** (1.0 / 3.0)
    return _call(_gen().sgpgen_rgg3d, n, radius, seed, name=f"rgg3d_{n}")


def chung_lu(n: int, alpha: float = 2.1, dmin: float = 12.5, dmax: float = 50000.0,
             wmax: int = 100, seed: int = 1) -> CSR:
    """Chung-Lu with Pareto(alpha, dmin) expected degrees capped at dmax and
    integer edge weights uniform in [1, wmax] (0 = unit weights)."""
    return _call(_gen().sgpgen_chunglu, n, alpha, dmin, dmax, wmax, seed, name=f"chunglu{n}")


def write_csr(path: str, g: CSR) -> None:
    """Write ``g`` in the reference's binary CSR format."""
    raw = _CSR()
    raw.n = g.n
    raw.m = g.m_directed
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(g.col, dtype=np.uint32)
    raw.row_ptr = rp.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    raw.col = col.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    if _gen().sgpgen_write_csr(path.encode(), ctypes.byref(raw)) != 0:
        raise OSError(f"could not write {path}")
