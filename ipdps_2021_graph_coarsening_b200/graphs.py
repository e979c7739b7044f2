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
        lib.sgpgen_mtx_lines.argtypes = [ctypes.c_void_p, ctypes.c_void_p, u64, i32, i32, ctypes.c_void_p, u64]
        lib.sgpgen_mtx_lines.restype = u64
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
    """Chung-Lu with Pareto expected degrees (shape alpha, scale dmin: mean
    alpha dmin / (alpha - 1), about 24 for the defaults) capped at dmax and
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


# ------------------------------------------------------------ MatrixMarket --
def mtx_text(u, v, rows: int, cols: int, field: str = "pattern", symmetry: str = "symmetric",
             comments=(), crlf: bool = False, nnz: Optional[int] = None) -> bytes:
    """MatrixMarket coordinate text of the 0-based entries ``(u[i], v[i])``
    in the given order: banner, ``%`` comment lines, size line, one line per
    entry (``real`` / ``integer`` fields get values the reader must skip)."""
    u = np.ascontiguousarray(u, dtype=np.uint32)
    v = np.ascontiguousarray(v, dtype=np.uint32)
    m = int(u.shape[0])
    vk = {"pattern": 0, "real": 1, "integer": 2}[field]
    nl = b"\r\n" if crlf else b"\n"
    head = f"%%MatrixMarket matrix coordinate {field} {symmetry}".encode() + nl
    for c in comments:
        head += b"%" + c.encode() + nl
    head += f"{rows} {cols} {m if nnz is None else nnz}".encode() + nl
    cap = m * 48 + 16
    buf = np.empty(cap, dtype=np.uint8)
    k = _gen().sgpgen_mtx_lines(u.ctypes.data, v.ctypes.data, m, vk, int(crlf), buf.ctypes.data, cap)
    if m and k == 0:
        raise RuntimeError("MatrixMarket formatting buffer too small")
    return head + buf[:k].tobytes()


def mtx_of(g: CSR, symmetry: str = "symmetric", field: str = "pattern", seed: Optional[int] = 0,
           dup_frac: float = 0.0, extra_vertices: int = 0, **kw) -> bytes:
    """A symmetric graph as MatrixMarket text.  ``symmetric`` stores the
    lower triangle (row > col), ``general`` every directed entry.  Lines are
    shuffled with ``seed`` (None: row order); ``dup_frac`` of them repeated;
    ``extra_vertices`` isolated vertices appended to the size line."""
    rows = np.repeat(np.arange(g.n, dtype=np.uint32), np.diff(g.row_ptr).astype(np.int64))
    cols = np.asarray(g.col, dtype=np.uint32)
    if symmetry == "symmetric":
        keep = rows > cols
        rows, cols = rows[keep], cols[keep]
    rng = np.random.default_rng(seed if seed is not None else 0)
    if dup_frac > 0:
        extra = rng.choice(rows.shape[0], int(dup_frac * rows.shape[0]), replace=True)
        rows, cols = np.concatenate([rows, rows[extra]]), np.concatenate([cols, cols[extra]])
    if seed is not None:
        p = rng.permutation(rows.shape[0])
        rows, cols = rows[p], cols[p]
    n = g.n + extra_vertices
    return mtx_text(rows, cols, n, n, field=field, symmetry=symmetry, **kw)


def batch_graphs(count: int = 2048, seed: int = 2048, lo: int = 1000, hi: int = 250000) -> list:
    """The batch configuration: vertex counts log-uniform in [lo, hi] from a
    fixed seed; even indices are near-square 2D grids with 10% of the vertices
    removed (largest component kept), odd ones Erdos-Renyi graphs of mean
    degree 8 (largest component), unit weights."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(int)
    out = []
    for i, s in enumerate(sizes):
        if i % 2 == 0:
            nx = int(math.sqrt(s))
            out.append(grid2d_holes(nx, max(2, int(s) // nx), seed=i + 1))
        else:
            out.append(erdos_renyi(int(s), 8.0, seed=i + 1))
    return out
