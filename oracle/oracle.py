"""ORACLE — test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import this module,
and only as the checker or as the timed CPU reference.  The product (graphine_b200/) never
imports it.

Two checkers:
* :class:`Restatement` - ctypes over ``libgre_oracle.so``, a C++ restatement of the reference
  engine loop and plugins (gre_oracle.cpp cites the reference lines it follows);
* :func:`run_reference` - runs the reference GRE engine itself, compiled from its headers by
  ``oracle/Makefile`` into ``oracle/_ref/`` (np = 1), through the harness drivers in
  ``oracle/ref_drivers/``.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgre_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} missing: run `make -C oracle restatement`")
        L = C.CDLL(LIB_PATH)
        P, U32, U64, I32, D = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double
        sig = {
            "oracle_load": (I32, [C.c_char_p, C.POINTER(P)]),
            "oracle_from_csr": (I32, [U64, U64, P, P, C.POINTER(P)]),
            "oracle_free": (None, [P]),
            "oracle_num_vertices": (U64, [P]),
            "oracle_num_arcs": (U64, [P]),
            "oracle_csr": (None, [P, P, P]),
            "oracle_pagerank": (I32, [P, I32, D, P, U32, P, P, U32, C.POINTER(U32)]),
            "oracle_ppr": (I32, [P, P, U32, D, U32, P]),
            "oracle_bfs": (I32, [P, U32, I32, P, P, P, U32, C.POINTER(U32)]),
            "oracle_bfs_many": (I32, [P, P, U32, I32, P]),
            "oracle_sssp": (I32, [P, U32, U64, P, P, P, U32, C.POINTER(U32)]),
            "oracle_sssp_many": (I32, [P, P, U32, U64, P, P]),
            "oracle_cc": (I32, [P, P, P, U32, C.POINTER(U32)]),
            "oracle_bc": (I32, [P, P, U32, P, C.POINTER(I32), P]),
            "oracle_bc_forward": (I32, [P, U32, P, P, P]),
            "oracle_pagerank_weighted": (I32, [P, P, P, D, U32, P]),
            "oracle_pagerank_adjoint": (I32, [P, P, P, P, D, U32, P, P, P]),
            "oracle_sssp_weight": (U32, [U64, U32, U32]),
            "oracle_pagerank_delta": (I32, [P, U32, P, P, U32, C.POINTER(U32)]),
            "oracle_sssp1": (I32, [P, U32, U64, P, P, P, P, U32, C.POINTER(U32)]),
            "oracle_count_in": (I32, [P, I32, U32, P, P, U32, C.POINTER(U32)]),
            "oracle_rmat": (I32, [U32, U32, U64, I32, C.POINTER(U64), C.POINTER(U64), C.POINTER(P), C.POINTER(P)]),
            "oracle_host_free": (None, [P]),
            "oracle_write_edgelists": (I32, [C.c_char_p, U64, U64, P, P, U32]),
            "oracle_write_roots": (I32, [C.c_char_p, P, U32]),
            "oracle_sssp_weights_csr": (None, [U64, U64, P, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


@dataclass
class Trace:
    supersteps: int = 0
    active: List[int] = field(default_factory=list)


class Restatement:
    """A graph loaded into the C++ restatement of the reference engine."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        self.n = int(lib().oracle_num_vertices(self._h))
        self.m = int(lib().oracle_num_arcs(self._h))

    @classmethod
    def load(cls, prefix: str) -> "Restatement":
        h = C.c_void_p()
        st = lib().oracle_load(prefix.encode(), C.byref(h))
        if st:
            raise RuntimeError(f"oracle_load({prefix}) failed: {st}")
        return cls(h.value)

    @classmethod
    def from_csr(cls, n: int, off: np.ndarray, col: np.ndarray) -> "Restatement":
        off = np.ascontiguousarray(off, dtype=np.uint64)
        col = np.ascontiguousarray(col, dtype=np.uint32)
        h = C.c_void_p()
        lib().oracle_from_csr(n, len(col), _p(off), _p(col), C.byref(h))
        return cls(h.value)

    def __del__(self):
        try:
            if self._h:
                lib().oracle_free(self._h)
        except Exception:
            pass

    def csr(self):
        off = np.empty(self.n + 1, dtype=np.uint64)
        col = np.empty(max(self.m, 1), dtype=np.uint32)
        lib().oracle_csr(self._h, _p(off), _p(col))
        return off, col[: self.m]

    @staticmethod
    def _trace(counts, nss) -> Trace:
        k = min(nss.value + 1, len(counts))
        return Trace(nss.value, [int(x) for x in counts[:k]])

    def pagerank(self, variant: int = 0, d: float = 0.85, supersteps: int = 20, teleport=None):
        pr = np.empty(self.n, dtype=np.float64)
        counts = np.zeros(1024, dtype=np.uint64)
        nss = C.c_uint32()
        tele = None if teleport is None else np.ascontiguousarray(teleport, dtype=np.float64)
        lib().oracle_pagerank(self._h, variant, d, _p(tele), supersteps, _p(pr), _p(counts), 1024, C.byref(nss))
        return pr, Trace(nss.value, [int(x) for x in counts[: nss.value]])

    def ppr(self, seeds, d: float = 0.85, supersteps: int = 20) -> np.ndarray:
        s = np.ascontiguousarray(seeds, dtype=np.uint32)
        out = np.empty(len(s) * self.n, dtype=np.float64)
        lib().oracle_ppr(self._h, _p(s), len(s), d, supersteps, _p(out))
        return out.reshape(len(s), self.n)

    def bfs(self, src: int, dir: int = 1):
        level = np.empty(self.n, dtype=np.int32)
        pred = np.empty(self.n, dtype=np.uint64)
        counts = np.zeros(1024, dtype=np.uint64)
        nss = C.c_uint32()
        lib().oracle_bfs(self._h, int(src), dir, _p(level), _p(pred), _p(counts), 1024, C.byref(nss))
        return level, pred, self._trace(counts, nss)

    def bfs_many(self, srcs, dir: int = 1) -> np.ndarray:
        s = np.ascontiguousarray(srcs, dtype=np.uint32)
        out = np.empty(len(s) * self.n, dtype=np.int32)
        lib().oracle_bfs_many(self._h, _p(s), len(s), dir, _p(out))
        return out.reshape(len(s), self.n)

    def sssp(self, src: int, wseed: int = 0, warc=None):
        dist = np.empty(self.n, dtype=np.uint32)
        counts = np.zeros(1024, dtype=np.uint64)
        nss = C.c_uint32()
        w = None if warc is None else np.ascontiguousarray(warc, dtype=np.uint32)
        lib().oracle_sssp(self._h, int(src), wseed, _p(w), _p(dist), _p(counts), 1024, C.byref(nss))
        return dist, self._trace(counts, nss)

    def sssp_many(self, srcs, wseed: int = 0, warc=None) -> np.ndarray:
        s = np.ascontiguousarray(srcs, dtype=np.uint32)
        out = np.empty(len(s) * self.n, dtype=np.uint32)
        w = None if warc is None else np.ascontiguousarray(warc, dtype=np.uint32)
        lib().oracle_sssp_many(self._h, _p(s), len(s), wseed, _p(w), _p(out))
        return out.reshape(len(s), self.n)

    def pagerank_delta(self, max_supersteps: int = 1024):
        pr = np.empty(self.n, dtype=np.float64)
        counts = np.zeros(1024, dtype=np.uint64)
        nss = C.c_uint32()
        lib().oracle_pagerank_delta(self._h, max_supersteps, _p(pr), _p(counts), 1024, C.byref(nss))
        return pr, self._trace(counts, nss)

    def sssp1(self, src: int, wseed: int = 0, warc=None):
        dist = np.empty(self.n, dtype=np.uint32)
        pred = np.empty(self.n, dtype=np.uint64)
        counts = np.zeros(1024, dtype=np.uint64)
        nss = C.c_uint32()
        w = None if warc is None else np.ascontiguousarray(warc, dtype=np.uint32)
        lib().oracle_sssp1(self._h, int(src), wseed, _p(w), _p(dist), _p(pred), _p(counts), 1024, C.byref(nss))
        return dist, pred, self._trace(counts, nss)

    def count_in(self, dir: int = 1, max_supersteps: int = 1):
        cn = np.empty(self.n, dtype=np.int32)
        counts = np.zeros(1024, dtype=np.uint64)
        nss = C.c_uint32()
        lib().oracle_count_in(self._h, dir, max_supersteps, _p(cn), _p(counts), 1024, C.byref(nss))
        return cn, self._trace(counts, nss)

    def cc(self):
        label = np.empty(self.n, dtype=np.uint64)
        counts = np.zeros(1024, dtype=np.uint64)
        nss = C.c_uint32()
        lib().oracle_cc(self._h, _p(label), _p(counts), 1024, C.byref(nss))
        return label, self._trace(counts, nss)

    def bc(self, srcs):
        s = np.ascontiguousarray(srcs, dtype=np.uint32)
        out = np.empty(self.n, dtype=np.float64)
        ovf = C.c_int(0)
        lib().oracle_bc(self._h, _p(s), len(s), _p(out), C.byref(ovf), None)
        return out, bool(ovf.value)

    def bc_forward(self, s: int):
        level = np.empty(self.n, dtype=np.int32)
        sigma = np.empty(self.n, dtype=np.float64)
        dep = np.empty(self.n, dtype=np.float64)
        lib().oracle_bc_forward(self._h, int(s), _p(level), _p(sigma), _p(dep))
        return level, sigma, dep

    def pagerank_weighted(self, warc, pers, d: float = 0.85, iters: int = 200) -> np.ndarray:
        w = np.ascontiguousarray(warc, dtype=np.float64)
        p = np.ascontiguousarray(pers, dtype=np.float64)
        r = np.empty(self.n, dtype=np.float64)
        lib().oracle_pagerank_weighted(self._h, _p(w), _p(p), d, iters, _p(r))
        return r

    def pagerank_adjoint(self, warc, r, c, d: float = 0.85, iters: int = 200):
        w = np.ascontiguousarray(warc, dtype=np.float64)
        r = np.ascontiguousarray(r, dtype=np.float64)
        c = np.ascontiguousarray(c, dtype=np.float64)
        lam = np.empty(self.n, dtype=np.float64)
        gp = np.empty(self.n, dtype=np.float64)
        gw = np.empty(self.m, dtype=np.float64)
        lib().oracle_pagerank_adjoint(self._h, _p(w), _p(r), _p(c), d, iters, _p(lam), _p(gp), _p(gw))
        return lam, gp, gw


def sssp_weight(wseed: int, u: int, v: int) -> int:
    return int(lib().oracle_sssp_weight(wseed, u, v))


def sssp_weights_csr(wseed: int, off: np.ndarray, col: np.ndarray) -> np.ndarray:
    """The harness SSSP weight of every arc of a CSR, in CSR order (uint32)."""
    off = np.ascontiguousarray(off, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    w = np.empty(max(len(col), 1), dtype=np.uint32)
    lib().oracle_sssp_weights_csr(wseed, len(off) - 1, _p(off), _p(col), _p(w))
    return w[: len(col)]


# ----------------------------------------------------------------------------------------------
# inputs, generated on the host without the product library (oracle/inputs.cpp)
# ----------------------------------------------------------------------------------------------
def rmat(scale: int, edgefactor: int = 16, seed: int = 1, symmetric: bool = True):
    """Seeded RMAT CSR: (n, off uint64[n+1], col uint32[m]); the same graph as the product's
    generator for the same arguments."""
    n, m = C.c_uint64(), C.c_uint64()
    po, pc = C.c_void_p(), C.c_void_p()
    st = lib().oracle_rmat(scale, edgefactor, seed, int(symmetric), C.byref(n), C.byref(m), C.byref(po), C.byref(pc))
    if st:
        raise RuntimeError(f"oracle_rmat({scale}, {edgefactor}, {seed}) failed: {st}")
    try:
        off = np.ctypeslib.as_array(C.cast(po, C.POINTER(C.c_uint64)), shape=(n.value + 1,)).copy()
        col = np.ctypeslib.as_array(C.cast(pc, C.POINTER(C.c_uint32)), shape=(max(m.value, 1),))[: m.value].copy()
    finally:
        lib().oracle_host_free(po)
        lib().oracle_host_free(pc)
    return n.value, off, col


def write_edgelists(prefix: str, n: int, off: np.ndarray, col: np.ndarray, nfiles: int = 4) -> None:
    off = np.ascontiguousarray(off, dtype=np.uint64)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    st = lib().oracle_write_edgelists(prefix.encode(), n, len(col), _p(off), _p(col) if len(col) else None, nfiles)
    if st:
        raise RuntimeError(f"oracle_write_edgelists({prefix}) failed: {st}")


def write_roots(prefix: str, roots) -> None:
    r = np.ascontiguousarray(roots, dtype=np.uint32)
    st = lib().oracle_write_roots(prefix.encode(), _p(r), len(r))
    if st:
        raise RuntimeError(f"oracle_write_roots({prefix}) failed: {st}")


def sample_sources(off: np.ndarray, k: int, seed: int) -> np.ndarray:
    """k distinct vertices with at least one arc, drawn with a seeded generator (sorted)."""
    deg = np.diff(off.astype(np.int64))
    cand = np.flatnonzero(deg > 0)
    if len(cand) <= k:
        return cand.astype(np.uint32)
    return np.sort(np.random.default_rng(seed).choice(cand, size=k, replace=False)).astype(np.uint32)


def reached_edges(off: np.ndarray, level: np.ndarray) -> int:
    """Graph500 numerator of a BFS/SSSP run on a symmetric graph: undirected edges with both
    endpoints reached (= half the arcs out of reached vertices)."""
    deg = np.diff(off.astype(np.int64))
    return int(deg[np.asarray(level) >= 0].sum() // 2)


# ----------------------------------------------------------------------------------------------
# the reference engine itself
# ----------------------------------------------------------------------------------------------
@dataclass
class RefRun:
    seconds: List[float]
    supersteps: List[int]
    active: List[List[int]]  # per run: the "Superstep-k: Number of active vertices...N" values
    stdout: str


def reference_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f"ref_{a}")) for a in ("pagerank", "bfs", "sssp", "cc", "bc"))


def _parse(stdout: str) -> RefRun:
    secs, sss, active, cur = [], [], [], []
    for line in stdout.splitlines():
        m = re.match(r"Superstep-(\d+): Number of active vertices\.\.\.(\d+)", line)
        if m:
            cur.append(int(m.group(2)))
            continue
        m = re.match(r"GRE_RUN (\S+) (\S+) (\S+)", line)
        if m:
            secs.append(float(m.group(2)))
            sss.append(int(m.group(3)))
            active.append(cur)
            cur = []
    return RefRun(secs, sss, active, stdout)


def run_reference(algo: str, prefix: str, *args, timeout: float = 600.0):
    """Run oracle/_ref/ref_<algo> on <prefix>; returns (array, RefRun)."""
    exe = os.path.join(REF_DIR, f"ref_{algo}")
    dtype = {"pagerank": np.float64, "bfs": np.int32, "sssp": np.uint32, "cc": np.uint64, "bc": np.float64,
             "sssp1": np.uint8, "countin": np.int32}[algo]
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.bin")
        p = subprocess.run([exe, prefix, out, *[str(a) for a in args]], capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"{exe} failed ({p.returncode}): {p.stderr[-2000:]}")
        arr = np.fromfile(out, dtype=dtype)
    return arr, _parse(p.stdout)
