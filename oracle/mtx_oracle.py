"""CPU restatement of the reference's MatrixMarket converter.

TEST INFRASTRUCTURE ONLY: the checker of the device converter
(``sgp_b200_mtx_read`` / ``sgp_b200_mtx_parse``), never part of it.  Pinned
byte for byte against the reference's own binaries (``oracle/_ref/mtx2csr``
and ``oracle/_ref/mtx2csr_large``, built from cmg/mtx2csr.cpp and
cmg/mtx2csr_large.cpp by ``oracle/Makefile``) in ``tests/test_mtx_oracle.py``.

Steps, each after the reference file cmg/mtx2csr.cpp:
  banner and comment lines            :49-83
  size line, symmetric / A+A^T /
  bipartite choice                    :87-104
  entries, both directions, self
  loops dropped unless bipartite      :105-128
  per-row sort + dedupe               :132-157
  largest component (first in vertex
  order on a tie), ascending ids      :166-264
  binary file                         :266-289
The reference's undefined cases (an id of 0 or beyond the size line, an entry
line that is not "i j ...", a symmetric banner on a non-square size line, a
later banner switching to "general") raise MtxError here, as the device path
fails on them; blank lines are skipped.
"""
from __future__ import annotations

import re

import numpy as np


class MtxError(ValueError):
    pass


_BLANK = b" \t\r\x0b\x0c"
_SIZE = re.compile(rb"[ \t\r\x0b\x0c]*([+-]?[0-9]+)[ \t\r\x0b\x0c]*([+-]?[0-9]+)(?:[ \t\r\x0b\x0c]*([+-]?[0-9]+))?")
_ENTRY = re.compile(rb"[ \t\r\x0b\x0c]*\+?([0-9]+)[ \t\r\x0b\x0c]*\+?([0-9]+)")


def _lines(text: bytes) -> list[bytes]:
    """getline over the text: a final '\\n' ends the last line."""
    parts = text.split(b"\n")
    if parts and parts[-1] == b"":
        parts.pop()
    return parts


def _banner(line: bytes) -> bool:
    """mtx2csr.cpp:53-79 -> whether the banner says "general"."""
    if b"coordinate" not in line:
        raise MtxError("banner does not say coordinate")
    return b"general" in line


def parse(text: bytes):
    """-> (n, u, v, info): the directed entries (both directions) the
    reference puts into its adjacency vectors, in file order."""
    lines = _lines(text)
    general = False
    i = 0
    size = None
    while i < len(lines):
        ln = lines[i]
        i += 1
        if ln[:1] == b"%":
            if ln[1:2] == b"%":
                general |= _banner(ln)
            continue
        if ln.split(b"\0")[0].strip(_BLANK + b"\0") == b"":
            continue
        mt = _SIZE.match(ln.split(b"\0")[0])   # sscanf "%ld %ld %ld"
        if not mt or int(mt.group(1)) < 0 or int(mt.group(2)) < 0:
            raise MtxError("bad size line")
        size = (int(mt.group(1)), int(mt.group(2)), int(mt.group(3)) if mt.group(3) else 0)
        break
    info = {"rows": 0, "cols": 0, "bipartite": 0, "lines": 0}
    if size is None:
        return 0, np.zeros(0, np.int64), np.zeros(0, np.int64), info
    rows, cols, _ = size
    if not general and rows != cols:
        raise MtxError("symmetric matrix with rows != cols")
    bip = rows != cols
    n = rows + cols if bip else rows
    shift = cols if bip else 0
    info.update(rows=rows, cols=cols, bipartite=int(bip), lines=len(lines) - i)
    us, vs = [], []
    for ln in lines[i:]:
        if ln[:1] == b"%":
            if ln[1:2] == b"%" and _banner(ln) and not bip:
                raise MtxError("a later banner switches to general")
            continue
        s = ln.split(b"\0")[0]
        if s.strip(_BLANK) == b"":
            continue
        mt = _ENTRY.match(s)
        if not mt:
            raise MtxError("entry line is not 'i j ...'")
        x, y = int(mt.group(1)), int(mt.group(2))
        if x == 0 or y == 0:
            raise MtxError("id 0")
        if x > rows or y > cols:
            raise MtxError("id beyond the size line")
        a, b = x - 1 + shift, y - 1
        if not bip and a == b:
            continue
        us.append(a)
        vs.append(b)
    u = np.asarray(us, dtype=np.int64)
    v = np.asarray(vs, dtype=np.int64)
    return n, np.concatenate([u, v]), np.concatenate([v, u]), info


def components(n: int, rp: np.ndarray, col: np.ndarray) -> np.ndarray:
    """Label of every vertex = the smallest vertex of its component (min-label
    propagation with pointer jumping)."""
    lab = np.arange(n, dtype=np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp).astype(np.int64))
    while True:
        new = lab.copy()
        if rows.size:
            np.minimum.at(new, rows, lab[col.astype(np.int64)])
        while True:
            j = new[new]
            if np.array_equal(j, new):
                break
            new = j
        if np.array_equal(new, lab):
            return lab
        lab = new


def convert(text: bytes):
    """-> (row_ptr uint32, col uint32, info): the reference's output graph."""
    n, u, v, info = parse(text)
    if n == 0:
        info.update(n_all=0, m_all=0, components=0, n=0, m=0)
        return np.zeros(1, np.uint32), np.zeros(0, np.uint32), info
    key = np.unique(u * n + v)
    su, sv = key // n, key % n
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum(np.bincount(su, minlength=n))
    lab = components(n, rp, sv)
    size = np.bincount(lab, minlength=n)
    roots = np.flatnonzero(lab == np.arange(n))
    best = roots[np.argmax(size[roots])]   # first root among the largest
    keep = lab == best
    newid = np.cumsum(keep) - 1
    deg = np.diff(rp)
    orp = np.zeros(int(keep.sum()) + 1, np.int64)
    orp[1:] = np.cumsum(deg[keep])
    sel = keep[su]
    ocol = newid[sv[sel]]
    info.update(n_all=n, m_all=int(key.size), components=int(roots.size), n=int(keep.sum()), m=int(ocol.size))
    return orp.astype(np.uint32), ocol.astype(np.uint32), info


def csr_bytes(rp: np.ndarray, col: np.ndarray, id_bytes: int = 4) -> bytes:
    """mtx2csr.cpp:276-288 (id_bytes 8: mtx2csr_large.cpp)."""
    dt = np.uint32 if id_bytes == 4 else np.uint64
    hdr = np.array([len(rp) - 1, len(col), 1, 0, 1, 0], dtype=np.int64)
    return hdr.tobytes() + rp.astype(dt).tobytes() + col.astype(dt).tobytes()
