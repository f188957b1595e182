"""Python mirror of the GRE superstep engine over the C ABI of libgre_gpu.so (include/gre_gpu.h).

The reference (NCIC-PARALLEL/Graphine, "GRE") is driven from C++ drivers (usr/test_*.cpp):
ingress a DistributedGraph from ``<prefix>.meta`` + ``<prefix>.edges.<i>``, build a plugin
(PageRank, BFS, SSSP, ConnectedComponents, BC Forward/Backward), run a SynchronousEngine.  This
module exposes the same steps with the same names where they exist:

* :class:`Graph` - ``DistributedGraph::ingress`` (Graph/DistributedGraph.hpp:153-172) and the
  graph queries (``get_num_masters``, ``get_num_edges``, ``getOutdegree``, ``loadEdgeProperty``).
* ``vc_*`` functions - the reference plugins on the device SynchronousEngine (per-superstep
  active counts as the reference prints them, Engine.hpp:392-398).
* ``pagerank``, ``bfs``, ``msbfs``, ``sssp``, ``cc``, ``bc``, ``ppr``, ``pagerank_weighted``,
  ``pagerank_adjoint`` - the B200 fast paths (same results).

Arrays: results come back as numpy arrays (host) unless ``out`` is given; ``out`` may be a
numpy array or a CUDA ``torch.Tensor`` (the library writes device memory in place).  Errors
raise :class:`GreError` carrying the status code (never a process exit).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgre_gpu.so")

# include/gre_gpu.h enums
GRE_SUCCESS, GRE_FAILURE, GRE_NOBUFFER, GRE_NULL, GRE_FINISHED, GRE_UNFINISHED = 0, 1, 2, 3, 4, 5
GRE_INITIALIZED, GRE_UNINITIALIZED, GRE_NOT_IMPLEMENTED, GRE_INVALID_ARG = 6, 7, 8, 9
GRE_IO_ERROR, GRE_CUDA_ERROR, GRE_OOM, GRE_TIMEOUT, GRE_NO_DEVICE = 10, 11, 12, 13, 14
Out, In, InOut = 0, 1, 2  # enum Dir (include/Types.hpp:33)
SYMMETRIC = 0x10
REORDER = 0x20
PR_REFERENCE, PR_ITER = 0, 1
MAX_RECORDED = 1024
XCHG_ALLGATHER, XCHG_ALLTOALL = 0, 1  # enum gre_exchange_kind
BATCH_BFS, BATCH_CC, BATCH_PAGERANK = 0, 2, 3  # enum gre_batch_algo


class BatchPageRankParams(C.Structure):
    _fields_ = [("variant", C.c_int), ("d", C.c_double), ("iters", C.c_uint32)]
# int (*gre_exchange_fn)(void* ctx, int kind, const void* send, void* recv, uint64_t bytes, void* stream)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p)


class GreError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {status_str(status)} ({status})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


class _Stats(C.Structure):
    _fields_ = [
        ("supersteps", C.c_uint32),
        ("n_recorded", C.c_uint32),
        ("arcs_traversed", C.c_uint64),
        ("traversed_edges", C.c_uint64),
        ("algo_bytes", C.c_uint64),
        ("device_ms", C.c_double),
        ("active", C.c_uint64 * MAX_RECORDED),
        ("plugin_value", C.c_double),
        ("plugin_count", C.c_uint64),
    ]


@dataclass
class Stats:
    """gre_stats: superstep count, per-superstep active vertices, traversal counters, time."""

    supersteps: int = 0
    active: List[int] = field(default_factory=list)
    arcs_traversed: int = 0
    traversed_edges: int = 0
    algo_bytes: int = 0
    device_ms: float = 0.0
    plugin_value: float = 0.0  # output_statistics: PageRank's sum of ranks
    plugin_count: int = 0      # output_statistics: CC's number of components

    @classmethod
    def _from(cls, s: _Stats) -> "Stats":
        return cls(s.supersteps, list(s.active[: s.n_recorded]), s.arcs_traversed, s.traversed_edges,
                   s.algo_bytes, s.device_ms, s.plugin_value, s.plugin_count)

    @property
    def gteps(self) -> float:
        return self.traversed_edges / (self.device_ms * 1e-3) / 1e9 if self.device_ms > 0 else 0.0

    @property
    def hbm_gbs(self) -> float:
        return self.algo_bytes / (self.device_ms * 1e-3) / 1e9 if self.device_ms > 0 else 0.0


_lib = None


def lib() -> C.CDLL:
    """Load libgre_gpu.so (fails loudly if the extension was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C graphine_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        P, U32, U64, I32, D = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double
        S = C.POINTER(_Stats)
        sig = {
            "gre_status_str": (C.c_char_p, [I32]),
            "gre_last_error": (C.c_char_p, []),
            "gre_device_count": (I32, [C.POINTER(I32)]),
            "gre_launch_count": (U64, []),
            "gre_graph_load": (I32, [C.c_char_p, U32, I32, C.POINTER(P)]),
            "gre_graph_load_parts": (I32, [C.c_char_p, U32, U32, I32, C.POINTER(P)]),
            "gre_graph_from_edges": (I32, [U64, U64, P, P, U32, I32, C.POINTER(P)]),
            "gre_graph_from_csr": (I32, [U64, U64, P, P, U32, I32, C.POINTER(P)]),
            "gre_graph_rmat": (I32, [U32, U32, U64, I32, I32, C.POINTER(P)]),
            "gre_graph_union": (I32, [P, U32, I32, C.POINTER(P), P]),
            "gre_graph_free": (I32, [P]),
            "gre_graph_reorder": (I32, [P]),
            "gre_graph_info": (I32, [P, C.POINTER(U64), C.POINTER(U64), C.POINTER(U32)]),
            "gre_row_schedule": (I32, [P, I32, C.POINTER(U32), C.POINTER(U64), C.POINTER(U64), C.POINTER(U64)]),
            "gre_graph_outdegree": (I32, [P, P]),
            "gre_graph_csr": (I32, [P, P, P]),
            "gre_graph_set_weights_u32": (I32, [P, P]),
            "gre_graph_set_weights_hash": (I32, [P, U64]),
            "gre_graph_set_weights_f64": (I32, [P, P]),
            "gre_vc_pagerank": (I32, [P, I32, U32, P, S]),
            "gre_vc_bfs": (I32, [P, U32, I32, P, P, S]),
            "gre_vc_sssp": (I32, [P, U32, U32, P, S]),
            "gre_vc_cc": (I32, [P, P, S]),
            "gre_vc_pagerank_delta": (I32, [P, U32, P, S]),
            "gre_vc_sssp1": (I32, [P, U32, U32, P, P, S]),
            "gre_vc_count_in": (I32, [P, I32, U32, P, S]),
            "gre_vc_bc": (I32, [P, P, U32, P, S]),
            "gre_pagerank": (I32, [P, I32, D, U32, P, S]),
            "gre_bfs": (I32, [P, P, U32, P, S]),
            "gre_bfs_noalloc": (I32, [P, U32, P, S]),
            "gre_msbfs": (I32, [P, P, U32, P, S]),
            "gre_bfs_multiroot": (I32, [P, P, U32, P, S]),
            "gre_sssp": (I32, [P, P, U32, P, S]),
            "gre_cc": (I32, [P, P, S]),
            "gre_bc": (I32, [P, P, U32, I32, P, S]),
            "gre_ppr": (I32, [P, P, U32, D, U32, I32, P, S]),
            "gre_pagerank_weighted": (I32, [P, D, P, D, U32, P, S]),
            "gre_pagerank_adjoint": (I32, [P, D, P, P, D, U32, P, P, P, S]),
            "gre_graph_batch_run": (I32, [P, U32, I32, P, P, S]),
            "gre_part_create": (I32, [P, U32, U32, C.POINTER(P)]),
            "gre_part_free": (I32, [P]),
            "gre_part_info": (I32, [P, C.POINTER(U64), C.POINTER(U64), C.POINTER(U64)]),
            "gre_nccl_unique_id": (I32, [P]),
            "gre_nccl_create": (I32, [P, U32, U32, I32, C.POINTER(P)]),
            "gre_nccl_free": (I32, [P]),
            "gre_nccl_exchange": (I32, [P, I32, P, P, U64, P]),
            "gre_part_layout": (I32, [U64, U32, C.POINTER(U64), P]),
            "gre_part_bfs": (I32, [P, U32, P, EXCHANGE_FN, P, S]),
            "gre_part_pagerank": (I32, [P, I32, D, U32, P, EXCHANGE_FN, P, S]),
            "gre_part_sssp": (I32, [P, U32, P, EXCHANGE_FN, P, S]),
            "gre_part_cc": (I32, [P, P, EXCHANGE_FN, P, S]),
            "gre_rmat_host": (I32, [U32, U32, U64, I32, C.POINTER(U64), C.POINTER(U64), C.POINTER(P), C.POINTER(P)]),
            "gre_host_free": (None, [P]),
            "gre_write_edgelists": (I32, [C.c_char_p, U64, U64, P, P, U32]),
            "gre_write_roots": (I32, [C.c_char_p, P, U32]),
            "gre_read_roots": (I32, [C.c_char_p, P, U32, C.POINTER(U32)]),
            "gre_sssp_weight": (U32, [U64, U32, U32]),
            "gre_partition_edges": (I32, [C.c_char_p, U32, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def status_str(status: int) -> str:
    return lib().gre_status_str(status).decode()


def last_error() -> str:
    return lib().gre_last_error().decode()


def _check(status: int, where: str) -> int:
    if status not in (GRE_SUCCESS, GRE_UNFINISHED):
        raise GreError(status, where, last_error())
    return status


def device_count() -> int:
    c = C.c_int(0)
    lib().gre_device_count(C.byref(c))
    return c.value


def launch_count() -> int:
    """Kernels launched by libgre_gpu.so so far in this process."""
    return int(lib().gre_launch_count())


# ----------------------------------------------------------------------------------------------
# buffers: numpy (host) or torch CUDA tensors (device)
# ----------------------------------------------------------------------------------------------
def _ptr(a) -> Optional[int]:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):  # torch.Tensor
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        if getattr(a, "is_cuda", False):
            import torch

            # the library orders its stream after the legacy default stream (PyTorch's default);
            # work the caller queued on another stream is finished here
            cur = torch.cuda.current_stream(a.device)
            if cur.cuda_stream != 0:
                cur.synchronize()
        return a.data_ptr()
    raise TypeError(f"unsupported buffer type {type(a)}")


def _as(a, dtype) -> np.ndarray:
    if hasattr(a, "data_ptr") and not isinstance(a, np.ndarray):
        return a  # torch tensor: passed through (host or device)
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def _out(out, count: int, dtype):
    if out is None:
        return np.empty(count, dtype=dtype)
    return out


# ----------------------------------------------------------------------------------------------
# Graph
# ----------------------------------------------------------------------------------------------
class Graph:
    """A device CSR (out-arcs) + CSC (in-arcs) graph; the DistributedGraph of one rank."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)
        n, m, f = C.c_uint64(), C.c_uint64(), C.c_uint32()
        _check(lib().gre_graph_info(self._h, C.byref(n), C.byref(m), C.byref(f)), "gre_graph_info")
        self.n, self.m, self.flags = n.value, m.value, f.value

    # --- construction -------------------------------------------------------------------------
    @classmethod
    def ingress(cls, prefix: str, dir: int = Out, symmetric: bool = False, device: int = 0,
                reorder: bool = False) -> "Graph":
        """DistributedGraph::ingress<dir>(comm, pool, prefix, "ascii", "edgelists")."""
        h = C.c_void_p()
        flags = dir | (SYMMETRIC if symmetric else 0) | (REORDER if reorder else 0)
        _check(lib().gre_graph_load(prefix.encode(), flags, device, C.byref(h)), "gre_graph_load")
        return cls(h.value)

    load = ingress

    @classmethod
    def load_parts(cls, prefix: str, nparts: int, dir: int = Out, symmetric: bool = False, device: int = 0,
                   reorder: bool = False) -> "Graph":
        """The reference's saved partitions <prefix>.part.<nparts>.<r> merged into one graph."""
        h = C.c_void_p()
        flags = dir | (SYMMETRIC if symmetric else 0) | (REORDER if reorder else 0)
        _check(lib().gre_graph_load_parts(prefix.encode(), nparts, flags, device, C.byref(h)), "gre_graph_load_parts")
        return cls(h.value)

    @classmethod
    def from_edges(cls, n: int, src, dst, dir: int = Out, symmetric: bool = False, device: int = 0,
                   reorder: bool = False) -> "Graph":
        s, d = _as(src, np.uint32), _as(dst, np.uint32)
        h = C.c_void_p()
        flags = dir | (SYMMETRIC if symmetric else 0) | (REORDER if reorder else 0)
        _check(lib().gre_graph_from_edges(n, len(s), _ptr(s), _ptr(d), flags, device, C.byref(h)), "gre_graph_from_edges")
        return cls(h.value)

    @classmethod
    def from_csr(cls, n: int, off, col, dir: int = Out, symmetric: bool = False, device: int = 0,
                 reorder: bool = False) -> "Graph":
        o, c = _as(off, np.uint64), _as(col, np.uint32)
        h = C.c_void_p()
        flags = dir | (SYMMETRIC if symmetric else 0) | (REORDER if reorder else 0)
        _check(lib().gre_graph_from_csr(n, len(c), _ptr(o), _ptr(c), flags, device, C.byref(h)), "gre_graph_from_csr")
        return cls(h.value)

    @classmethod
    def rmat(cls, scale: int, edgefactor: int = 16, seed: int = 1, symmetric: bool = True, device: int = 0,
             reorder: bool = False) -> "Graph":
        h = C.c_void_p()
        _check(lib().gre_graph_rmat(scale, edgefactor, seed, int(symmetric), device, C.byref(h)), "gre_graph_rmat")
        g = cls(h.value)
        if reorder:
            g.reorder()
        return g

    def reorder(self) -> None:
        """Relabel the stored graph by decreasing degree (invisible to callers)."""
        _check(lib().gre_graph_reorder(self._h), "gre_graph_reorder")
        n, m, f = C.c_uint64(), C.c_uint64(), C.c_uint32()
        _check(lib().gre_graph_info(self._h, C.byref(n), C.byref(m), C.byref(f)), "gre_graph_info")
        self.flags = f.value

    @classmethod
    def union(cls, graphs: Sequence["Graph"], device: int = 0):
        """Block-diagonal union; returns (graph, vertex_offset[k+1])."""
        arr = (C.c_void_p * len(graphs))(*[g._h.value for g in graphs])
        offs = np.zeros(len(graphs) + 1, dtype=np.uint64)
        h = C.c_void_p()
        _check(lib().gre_graph_union(arr, len(graphs), device, C.byref(h), _ptr(offs)), "gre_graph_union")
        return cls(h.value), offs

    def free(self) -> None:
        if self._h:
            lib().gre_graph_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # --- queries (DistributedGraph) ------------------------------------------------------------
    def get_num_masters(self) -> int:
        return self.n

    def get_num_edges(self) -> int:
        return self.m

    @property
    def symmetric(self) -> bool:
        return bool(self.flags & SYMMETRIC)

    def getOutdegree(self, out=None):
        out = _out(out, self.n, np.uint32)
        _check(lib().gre_graph_outdegree(self._h, _ptr(out)), "gre_graph_outdegree")
        return out

    def row_schedule(self, incoming: bool = True):
        """(lane_arcs, cta_min, hub_chunk, seg_window) of the degree bins, tuned on first use."""
        a, c, h, w = C.c_uint32(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(lib().gre_row_schedule(self._h, int(incoming), C.byref(a), C.byref(c), C.byref(h), C.byref(w)),
               "gre_row_schedule")
        return a.value, c.value, h.value, w.value

    def csr(self):
        off = np.empty(self.n + 1, dtype=np.uint64)
        col = np.empty(max(self.m, 1), dtype=np.uint32)
        _check(lib().gre_graph_csr(self._h, _ptr(off), _ptr(col)), "gre_graph_csr")
        return off, col[: self.m]

    # --- edge properties (DistributedGraph::loadEdgeProperty) ----------------------------------
    def loadEdgeProperty(self, w) -> None:
        w = _as(w, np.uint32)
        _check(lib().gre_graph_set_weights_u32(self._h, _ptr(w)), "gre_graph_set_weights_u32")

    def set_weights_hash(self, wseed: int) -> None:
        _check(lib().gre_graph_set_weights_hash(self._h, wseed), "gre_graph_set_weights_hash")

    def set_weights_f64(self, w) -> None:
        w = _as(w, np.float64)
        _check(lib().gre_graph_set_weights_f64(self._h, _ptr(w)), "gre_graph_set_weights_f64")


def _stats() -> _Stats:
    return _Stats()


def _srcs(srcs) -> np.ndarray:
    return _as(np.atleast_1d(np.asarray(srcs)) if not hasattr(srcs, "data_ptr") else srcs, np.uint32)


# ----------------------------------------------------------------------------------------------
# reference-semantics engine (plugins on the device SynchronousEngine)
# ----------------------------------------------------------------------------------------------
def vc_pagerank(g: Graph, variant: int = PR_REFERENCE, max_supersteps: int = 10, out=None):
    out = _out(out, g.n, np.float64)
    st = _stats()
    _check(lib().gre_vc_pagerank(g._h, variant, max_supersteps, _ptr(out), C.byref(st)), "gre_vc_pagerank")
    return out, Stats._from(st)


def vc_bfs(g: Graph, src: int, dir: int = In, pred=None, level=None):
    pred = _out(pred, g.n, np.uint64)
    level = _out(level, g.n, np.int32)
    st = _stats()
    _check(lib().gre_vc_bfs(g._h, int(src), dir, _ptr(pred), _ptr(level), C.byref(st)), "gre_vc_bfs")
    return pred, level, Stats._from(st)


def vc_sssp(g: Graph, src: int, max_supersteps: int = 1024, out=None):
    out = _out(out, g.n, np.uint32)
    st = _stats()
    status = _check(lib().gre_vc_sssp(g._h, int(src), max_supersteps, _ptr(out), C.byref(st)), "gre_vc_sssp")
    return out, Stats._from(st), status


def vc_pagerank_delta(g: Graph, max_supersteps: int = 1024, out=None):
    """PageRank_delta on the device engine; returns (pr, stats, status) (GRE_UNFINISHED if capped)."""
    out = _out(out, g.n, np.float64)
    st = _stats()
    status = lib().gre_vc_pagerank_delta(g._h, max_supersteps, _ptr(out), C.byref(st))
    if status not in (GRE_SUCCESS, GRE_UNFINISHED):
        _check(status, "gre_vc_pagerank_delta")
    return out, Stats._from(st), status


def vc_sssp1(g: Graph, src: int, max_supersteps: int = 1024):
    """SSSP1 (distances + predecessors); returns (dist, pred, stats, status)."""
    dist = np.empty(g.n, np.uint32)
    pred = np.empty(g.n, np.uint64)
    st = _stats()
    status = lib().gre_vc_sssp1(g._h, src, max_supersteps, _ptr(dist), _ptr(pred), C.byref(st))
    if status not in (GRE_SUCCESS, GRE_UNFINISHED):
        _check(status, "gre_vc_sssp1")
    return dist, pred, Stats._from(st), status


def vc_count_in(g: Graph, dir: int = In, max_supersteps: int = 1, out=None):
    out = _out(out, g.n, np.int32)
    st = _stats()
    _check(lib().gre_vc_count_in(g._h, dir, max_supersteps, _ptr(out), C.byref(st)), "gre_vc_count_in")
    return out, Stats._from(st)


def vc_cc(g: Graph, out=None):
    out = _out(out, g.n, np.uint32)
    st = _stats()
    _check(lib().gre_vc_cc(g._h, _ptr(out), C.byref(st)), "gre_vc_cc")
    return out, Stats._from(st)


def vc_bc(g: Graph, srcs, out=None):
    s = _srcs(srcs)
    out = _out(out, g.n, np.float64)
    st = _stats()
    _check(lib().gre_vc_bc(g._h, _ptr(s), len(s), _ptr(out), C.byref(st)), "gre_vc_bc")
    return out, Stats._from(st)


# ----------------------------------------------------------------------------------------------
# fast paths
# ----------------------------------------------------------------------------------------------
def pagerank(g: Graph, variant: int = PR_ITER, d: float = 0.85, iters: int = 20, out=None):
    out = _out(out, g.n, np.float64)
    st = _stats()
    _check(lib().gre_pagerank(g._h, variant, d, iters, _ptr(out), C.byref(st)), "gre_pagerank")
    return out, Stats._from(st)


def bfs(g: Graph, srcs, out=None):
    s = _srcs(srcs)
    out = _out(out, len(s) * g.n, np.int32)
    st = _stats()
    _check(lib().gre_bfs(g._h, _ptr(s), len(s), _ptr(out), C.byref(st)), "gre_bfs")
    return out, Stats._from(st)


def msbfs(g: Graph, srcs, out=None):
    s = _srcs(srcs)
    out = _out(out, len(s) * g.n, np.int32)
    st = _stats()
    _check(lib().gre_msbfs(g._h, _ptr(s), len(s), _ptr(out), C.byref(st)), "gre_msbfs")
    return out, Stats._from(st)


def bfs_multiroot(g: Graph, roots, out=None):
    s = _srcs(roots)
    out = _out(out, g.n, np.int32)
    st = _stats()
    _check(lib().gre_bfs_multiroot(g._h, _ptr(s), len(s), _ptr(out), C.byref(st)), "gre_bfs_multiroot")
    return out, Stats._from(st)


def sssp(g: Graph, srcs, out=None):
    s = _srcs(srcs)
    out = _out(out, len(s) * g.n, np.uint32)
    st = _stats()
    _check(lib().gre_sssp(g._h, _ptr(s), len(s), _ptr(out), C.byref(st)), "gre_sssp")
    return out, Stats._from(st)


def cc(g: Graph, out=None):
    out = _out(out, g.n, np.uint32)
    st = _stats()
    _check(lib().gre_cc(g._h, _ptr(out), C.byref(st)), "gre_cc")
    return out, Stats._from(st)


def bc(g: Graph, srcs, batched: bool = True, out=None):
    s = _srcs(srcs)
    out = _out(out, g.n, np.float64)
    st = _stats()
    _check(lib().gre_bc(g._h, _ptr(s), len(s), int(batched), _ptr(out), C.byref(st)), "gre_bc")
    return out, Stats._from(st)


def ppr(g: Graph, seeds, d: float = 0.85, iters: int = 20, batched: bool = True, out=None):
    s = _srcs(seeds)
    out = _out(out, len(s) * g.n, np.float64)
    st = _stats()
    _check(lib().gre_ppr(g._h, _ptr(s), len(s), d, iters, int(batched), _ptr(out), C.byref(st)), "gre_ppr")
    return out, Stats._from(st)


def pagerank_weighted(g: Graph, d: float = 0.85, pers=None, tol: float = 1e-14, max_iters: int = 1000, out=None):
    p = None if pers is None else _as(pers, np.float64)
    out = _out(out, g.n, np.float64)
    st = _stats()
    status = _check(lib().gre_pagerank_weighted(g._h, d, _ptr(p), tol, max_iters, _ptr(out), C.byref(st)),
                    "gre_pagerank_weighted")
    return out, Stats._from(st), status


def pagerank_adjoint(g: Graph, r, c, d: float = 0.85, tol: float = 1e-14, max_iters: int = 1000, lam=None,
                     grad_pers=None, grad_w=None):
    r, c = _as(r, np.float64), _as(c, np.float64)
    lam = _out(lam, g.n, np.float64)
    grad_pers = _out(grad_pers, g.n, np.float64)
    grad_w = _out(grad_w, g.m, np.float64)
    st = _stats()
    status = _check(lib().gre_pagerank_adjoint(g._h, d, _ptr(r), _ptr(c), tol, max_iters, _ptr(lam), _ptr(grad_pers),
                                               _ptr(grad_w), C.byref(st)), "gre_pagerank_adjoint")
    return lam, grad_pers, grad_w, Stats._from(st), status


# ----------------------------------------------------------------------------------------------
# host utilities (no GPU)
# ----------------------------------------------------------------------------------------------
def graph_batch_run(graphs: Sequence[Graph], algo: int, roots=None, variant: int = PR_ITER, d: float = 0.85,
                    iters: int = 20, outs=None):
    """gre_graph_batch_run: one algorithm over k graphs in one launch sequence; returns the
    per-graph result arrays (member ids) and the stats of the run over their union."""
    k = len(graphs)
    dt = np.float64 if algo == BATCH_PAGERANK else (np.int32 if algo == BATCH_BFS else np.uint32)
    outs = [np.empty(g.n, dtype=dt) for g in graphs] if outs is None else list(outs)
    arr = (C.c_void_p * k)(*[g._h.value for g in graphs])
    optr = (C.c_void_p * k)(*[_ptr(o) for o in outs])
    keep = None
    if algo == BATCH_BFS:
        keep = _as(roots, np.uint32)
        par = _ptr(keep)
    elif algo == BATCH_PAGERANK:
        keep = BatchPageRankParams(variant, d, iters)
        par = C.addressof(keep)
    else:
        par = None
    st = _stats()
    _check(lib().gre_graph_batch_run(arr, k, algo, par, optr, C.byref(st)), "gre_graph_batch_run")
    return outs, Stats._from(st)


def rmat_host(scale: int, edgefactor: int = 16, seed: int = 1, symmetric: bool = True):
    """Seeded RMAT CSR on the host: (n, row_off uint64[n+1], col uint32[m])."""
    n, m = C.c_uint64(), C.c_uint64()
    po, pc = C.c_void_p(), C.c_void_p()
    _check(lib().gre_rmat_host(scale, edgefactor, seed, int(symmetric), C.byref(n), C.byref(m), C.byref(po), C.byref(pc)),
           "gre_rmat_host")
    try:
        off = np.ctypeslib.as_array(C.cast(po, C.POINTER(C.c_uint64)), shape=(n.value + 1,)).copy()
        col = np.ctypeslib.as_array(C.cast(pc, C.POINTER(C.c_uint32)), shape=(max(m.value, 1),))[: m.value].copy()
    finally:
        lib().gre_host_free(po)
        lib().gre_host_free(pc)
    return n.value, off, col


def write_edgelists(prefix: str, n: int, off, col, nfiles: int = 4) -> None:
    o, c = _as(off, np.uint64), _as(col, np.uint32)
    _check(lib().gre_write_edgelists(prefix.encode(), n, len(c), _ptr(o), _ptr(c) if len(c) else None, nfiles),
           "gre_write_edgelists")


def partition_edges(prefix: str, nparts: int) -> np.ndarray:
    """Split <prefix>.edges.<i> into <prefix>.part.<nparts>.<r> (and the .outdegree / .scatterMap
    files) as the reference's offline partitioner does; returns the edges per part.  Host only."""
    counts = np.zeros(nparts, np.uint64)
    _check(lib().gre_partition_edges(prefix.encode(), nparts, _ptr(counts)), "gre_partition_edges")
    return counts


def write_roots(prefix: str, roots) -> None:
    r = _as(roots, np.uint32)
    _check(lib().gre_write_roots(prefix.encode(), _ptr(r), len(r)), "gre_write_roots")


def read_roots(prefix: str) -> np.ndarray:
    cnt = C.c_uint32()
    _check(lib().gre_read_roots(prefix.encode(), None, 0, C.byref(cnt)), "gre_read_roots")
    out = np.empty(max(cnt.value, 1), dtype=np.uint32)
    _check(lib().gre_read_roots(prefix.encode(), _ptr(out), cnt.value, C.byref(cnt)), "gre_read_roots")
    return out[: cnt.value]


def sssp_weight(wseed: int, u: int, v: int) -> int:
    return lib().gre_sssp_weight(wseed, u, v)


def sample_sources(off: np.ndarray, k: int, seed: int) -> np.ndarray:
    """k distinct vertices with at least one arc, drawn with a seeded generator."""
    n = len(off) - 1
    deg = np.diff(off.astype(np.int64))
    cand = np.flatnonzero(deg > 0)
    rng = np.random.default_rng(seed)
    if len(cand) <= k:
        return cand.astype(np.uint32)
    return np.sort(rng.choice(cand, size=k, replace=False)).astype(np.uint32)
