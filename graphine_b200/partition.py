"""1D-partitioned single-source paths (BFS, PageRank, SSSP, CC): one graph split by vertex over
ranks, one GPU per rank.

The reference spreads one graph over MPI ranks (vertex placement, GraphIngress.hpp:1126-1450)
and runs every superstep as sync scatters -> local compute -> sync combiners -> apply
(Engine.hpp:273-374).  ``gre_part_*`` of the C ABI do the same on GPUs with a fixed placement
(vertices dealt to ranks one by one in snake order, see :func:`layout`): each rank keeps the
in- and out-arcs of its own vertices, and the exchanges are

* PageRank: an all-gather of the owners' contributions every superstep (8 bytes per vertex);
* BFS bottom-up level: an all-gather of the owners' frontier bits (n/8 bytes);
* BFS top-down level: an all-to-all of candidate bitmaps (each owner ORs the blocks it gets),
* SSSP superstep: an all-to-all of candidate distances (each owner keeps the smallest offer),
* CC superstep: an all-gather of the labels (4 bytes per vertex),

plus a 32-byte all-gather of the level counters.  The library calls back into the host for each
collective (``gre_exchange_fn``); this module supplies three implementations:

* :class:`NcclExchange` - the library's own NCCL communicator (``gre_nccl_exchange``): the
  collectives are enqueued by the library on the part's stream, no Python in the loop.  The
  default for multi-GPU runs.
* :class:`TorchExchange` - the collectives of a ``torch.distributed`` process group: NCCL on
  the part's own CUDA stream for device buffers; host buffers over any backend (gloo).
* :class:`LocalExchange` - P parts in one process, one thread each (all on one GPU or spread
  over several): a collective is a host barrier plus device copies, so no kernel ever waits for
  another.

Every rank returns all n results in caller vertex order.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import Callable, List, Optional, Tuple

import numpy as np

from . import gre as G

ALLGATHER, ALLTOALL = G.XCHG_ALLGATHER, G.XCHG_ALLTOALL

# exchange(kind, send_ptr, recv_ptr, nbytes, stream_ptr) -> None; raises on failure
Exchange = Callable[[int, int, int, int, int], None]


def layout(n: int, nparts: int) -> Tuple[int, np.ndarray]:
    """(L, index): slots per rank and the exchange index of every internal vertex id.

    Round r = v // P and t = v % P give vertex v the rank p = t on even rounds and P - 1 - t on
    odd ones (snake order); it is slot r of that rank, exchange index p * L + r, with
    L = 64 * ceil(ceil(n / P) / 64) slots per rank (whole bitmap words).  Internal ids are in
    decreasing degree on a relabelled graph, so every rank gets the same mix of degrees."""
    P = int(nparts)
    per = (n + P - 1) // P
    L = 64 * max(1, (per + 63) // 64)
    v = np.arange(n, dtype=np.int64)
    r, t = v // P, v % P
    p = np.where(r & 1, P - 1 - t, t)
    return L, (p * L + r).astype(np.int64)


# ----------------------------------------------------------------------------------------------
# raw buffers as tensors
# ----------------------------------------------------------------------------------------------
class _CudaBytes:
    """A device byte range viewed through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 2, "strides": None}


def device_bytes(ptr: int, nbytes: int):
    import torch

    return torch.as_tensor(_CudaBytes(ptr, nbytes), device="cuda")


def host_bytes(ptr: int, nbytes: int):
    import torch

    return torch.from_numpy(np.ctypeslib.as_array((C.c_uint8 * int(nbytes)).from_address(int(ptr))))


class TorchExchange:
    """Collectives of a torch.distributed process group.

    ``memory="device"`` (the library's buffers): with NCCL the collective is enqueued on the
    part's stream (the stream waits for it before the next kernel); with another backend the
    bytes are staged through host memory.  ``memory="host"``: the pointers are host memory."""

    def __init__(self, group=None, memory: str = "device"):
        if memory not in ("device", "host"):
            raise ValueError("memory must be 'device' or 'host'")
        import torch.distributed as dist

        self.group = group
        self.memory = memory
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)

    def _collective(self, kind: int, send, recv) -> None:
        import torch.distributed as dist

        if kind == ALLGATHER:
            dist.all_gather_into_tensor(recv, send, group=self.group)
        elif kind == ALLTOALL:
            dist.all_to_all_single(recv, send, group=self.group)
        else:
            raise ValueError(f"unknown exchange kind {kind}")

    def __call__(self, kind: int, send_ptr: int, recv_ptr: int, nbytes: int, stream_ptr: int) -> None:
        import torch
        import torch.distributed as dist

        world = self.world
        sbytes = nbytes * (world if kind == ALLTOALL else 1)
        if self.memory == "host":
            self._collective(kind, host_bytes(send_ptr, sbytes), host_bytes(recv_ptr, nbytes * world))
            return
        stream = torch.cuda.ExternalStream(stream_ptr)
        send, recv = device_bytes(send_ptr, sbytes), device_bytes(recv_ptr, nbytes * world)
        if dist.get_backend(self.group) == "nccl":
            with torch.cuda.stream(stream):
                self._collective(kind, send, recv)
            return
        stream.synchronize()
        hs, hr = send.cpu(), torch.empty(nbytes * world, dtype=torch.uint8)
        self._collective(kind, hs, hr)
        with torch.cuda.stream(stream):
            recv.copy_(hr)
        stream.synchronize()


class NcclExchange:
    """A communicator of the library (gre_nccl_create) over the ranks of `group`: rank 0 makes
    the NCCL unique id and the process group carries it to the others (any backend).  Without
    an initialised process group this is a one-rank communicator.  Passed to :class:`Part`
    calls, the library calls ``gre_nccl_exchange`` itself."""

    def __init__(self, group=None, device: Optional[int] = None):
        import torch
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.world = 0, 1
        uid = (C.c_uint8 * 128)()
        if self.rank == 0:
            G._check(G.lib().gre_nccl_unique_id(uid), "gre_nccl_unique_id")
        if self.world > 1:
            box = [bytes(uid)]
            src = dist.get_global_rank(group, 0) if group is not None else 0
            dist.broadcast_object_list(box, src=src, group=group)
            C.memmove(uid, box[0], 128)
        dev = torch.cuda.current_device() if device is None else int(device)
        h = C.c_void_p()
        G._check(G.lib().gre_nccl_create(uid, self.world, self.rank, dev, C.byref(h)), "gre_nccl_create")
        self._h = h
        self.c_fn = G.EXCHANGE_FN(C.cast(G.lib().gre_nccl_exchange, C.c_void_p).value)

    @property
    def c_ctx(self):
        return self._h

    def free(self) -> None:
        if self._h:
            G.lib().gre_nccl_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class LocalExchange:
    """The ranks of one process: part r is driven by thread r, all collectives meet at a host
    barrier.  A rank synchronises its stream, publishes its send buffer, waits for all P, copies
    what it receives on its own stream, synchronises, and waits again so that no send buffer
    changes while another rank still reads it.  A rank that does not arrive within `timeout`
    seconds breaks the barrier: every waiting rank's call then fails (GRE_FAILURE)."""

    def __init__(self, nparts: int, timeout: float = 120.0):
        self.P = int(nparts)
        self.barrier = threading.Barrier(self.P, timeout=timeout)
        self.sends: List[int] = [0] * self.P

    def for_rank(self, rank: int) -> Exchange:
        return lambda kind, s, r, nb, st: self._run(rank, kind, s, r, nb, st)

    def abort(self) -> None:
        self.barrier.abort()

    def _run(self, rank: int, kind: int, send_ptr: int, recv_ptr: int, nbytes: int, stream_ptr: int) -> None:
        import torch

        stream = torch.cuda.ExternalStream(stream_ptr)
        stream.synchronize()
        self.sends[rank] = send_ptr
        self.barrier.wait()
        with torch.cuda.stream(stream):
            dst = device_bytes(recv_ptr, nbytes * self.P)
            for q in range(self.P):
                off = rank * nbytes if kind == ALLTOALL else 0
                dst[q * nbytes:(q + 1) * nbytes].copy_(device_bytes(self.sends[q] + off, nbytes))
        stream.synchronize()
        self.barrier.wait()


# ----------------------------------------------------------------------------------------------
# parts
# ----------------------------------------------------------------------------------------------
class _Callback:
    """A Python exchange as a gre_exchange_fn; the first exception is kept and re-raised."""

    def __init__(self, fn: Exchange):
        self.error: Optional[BaseException] = None

        def tramp(ctx, kind, send, recv, nbytes, stream):
            try:
                fn(int(kind), int(send or 0), int(recv or 0), int(nbytes), int(stream or 0))
                return 0
            except BaseException as e:  # noqa: BLE001 - reported after the C call returns
                if self.error is None:
                    self.error = e
                return 1

        self.c = G.EXCHANGE_FN(tramp)

    def check(self, status: int, where: str) -> None:
        if self.error is not None and status != G.GRE_SUCCESS:
            raise G.GreError(status, where, f"exchange failed: {self.error!r}") from self.error
        G._check(status, where)


class Part:
    """Rank `rank` of `nparts`: the rows of its slots of graph `g` (g may be freed after)."""

    def __init__(self, g: "G.Graph", nparts: int, rank: int):
        h = C.c_void_p()
        G._check(G.lib().gre_part_create(g._h, int(nparts), int(rank), C.byref(h)), "gre_part_create")
        self._h = h
        self.n, self.nparts, self.rank = g.n, int(nparts), int(rank)
        L, ai, ao = C.c_uint64(), C.c_uint64(), C.c_uint64()
        G._check(G.lib().gre_part_info(self._h, C.byref(L), C.byref(ai), C.byref(ao)), "gre_part_info")
        self.slots, self.arcs_in, self.arcs_out = L.value, ai.value, ao.value

    def free(self) -> None:
        if self._h:
            G.lib().gre_part_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @staticmethod
    def _exchange(exchange):
        """(function pointer, ctx, callback): a library exchange (NcclExchange) is passed as is;
        a Python callable goes through a ctypes trampoline."""
        if hasattr(exchange, "c_fn"):
            return exchange.c_fn, exchange.c_ctx, None
        cb = _Callback(exchange)
        return cb.c, None, cb

    def bfs(self, src: int, exchange, out=None):
        """Levels of all n vertices (caller order) from caller vertex `src`; -1 unreached."""
        out = G._out(out, self.n, np.int32)
        st = G._stats()
        cfn, ctx, cb = self._exchange(exchange)
        status = G.lib().gre_part_bfs(self._h, int(src), G._ptr(out), cfn, ctx, C.byref(st))
        (cb.check if cb is not None else G._check)(status, "gre_part_bfs")
        return out, G.Stats._from(st)

    def sssp(self, src: int, exchange, out=None):
        """Distances of all n vertices (caller order) from caller vertex `src` (0xffffffff
        unreached), with the uint32 weights the graph had when the part was made."""
        out = G._out(out, self.n, np.uint32)
        st = G._stats()
        cfn, ctx, cb = self._exchange(exchange)
        status = G.lib().gre_part_sssp(self._h, int(src), G._ptr(out), cfn, ctx, C.byref(st))
        (cb.check if cb is not None else G._check)(status, "gre_part_sssp")
        return out, G.Stats._from(st)

    def cc(self, exchange, out=None):
        """Component labels of all n vertices (smallest caller id of the weak component)."""
        out = G._out(out, self.n, np.uint32)
        st = G._stats()
        cfn, ctx, cb = self._exchange(exchange)
        status = G.lib().gre_part_cc(self._h, G._ptr(out), cfn, ctx, C.byref(st))
        (cb.check if cb is not None else G._check)(status, "gre_part_cc")
        return out, G.Stats._from(st)

    def pagerank(self, exchange, variant: int = G.PR_ITER, d: float = 0.85, iters: int = 20, out=None):
        """PageRank of all n vertices (caller order), as :func:`graphine_b200.gre.pagerank`."""
        out = G._out(out, self.n, np.float64)
        st = G._stats()
        cfn, ctx, cb = self._exchange(exchange)
        status = G.lib().gre_part_pagerank(self._h, variant, d, int(iters), G._ptr(out), cfn, ctx, C.byref(st))
        (cb.check if cb is not None else G._check)(status, "gre_part_pagerank")
        return out, G.Stats._from(st)


def library_layout(n: int, nparts: int) -> Tuple[int, np.ndarray]:
    """:func:`layout` as the library computes it (gre_part_layout, host code)."""
    L = C.c_uint64()
    idx = np.empty(n, dtype=np.uint32)
    G._check(G.lib().gre_part_layout(int(n), int(nparts), C.byref(L), G._ptr(idx)), "gre_part_layout")
    return L.value, idx.astype(np.int64)


def run_local(g: "G.Graph", nparts: int, job: Callable[[Part, Exchange], object]) -> list:
    """Run `job(part, exchange)` for parts 0..nparts-1 of `g`, one thread each (LocalExchange),
    all on g's device.  Returns the jobs' results in rank order; re-raises the first failure
    after every thread has ended."""
    import torch

    parts = [Part(g, nparts, r) for r in range(nparts)]
    x = LocalExchange(nparts)
    results: list = [None] * nparts
    errors: list = [None] * nparts
    device = torch.cuda.current_device()

    def work(r: int) -> None:
        try:
            torch.cuda.set_device(device)
            results[r] = job(parts[r], x.for_rank(r))
        except BaseException as e:  # noqa: BLE001
            errors[r] = e
            x.abort()

    threads = [threading.Thread(target=work, args=(r,)) for r in range(nparts)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for p in parts:
        p.free()
    for e in errors:
        if e is not None:
            raise e
    return results


def bfs(g: "G.Graph", src: int, group=None, exchange=None):
    """BFS levels over the ranks of `group`: this rank's part of g, the exchange the library's
    NCCL communicator (or `exchange`); every rank returns all n levels."""
    x = exchange if exchange is not None else NcclExchange(group)
    p = Part(g, x.world, x.rank)
    try:
        return p.bfs(src, x)
    finally:
        p.free()
        if exchange is None:
            x.free()


def sssp(g: "G.Graph", src: int, group=None, exchange=None):
    """SSSP distances over the ranks of `group` (as :func:`bfs`)."""
    x = exchange if exchange is not None else NcclExchange(group)
    p = Part(g, x.world, x.rank)
    try:
        return p.sssp(src, x)
    finally:
        p.free()
        if exchange is None:
            x.free()


def cc(g: "G.Graph", group=None, exchange=None):
    """Component labels over the ranks of `group` (as :func:`bfs`)."""
    x = exchange if exchange is not None else NcclExchange(group)
    p = Part(g, x.world, x.rank)
    try:
        return p.cc(x)
    finally:
        p.free()
        if exchange is None:
            x.free()


def pagerank(g: "G.Graph", variant: int = G.PR_ITER, d: float = 0.85, iters: int = 20, group=None, exchange=None):
    """PageRank over the ranks of `group` (as :func:`bfs`); every rank returns all n values."""
    x = exchange if exchange is not None else NcclExchange(group)
    p = Part(g, x.world, x.rank)
    try:
        return p.pagerank(x, variant, d, iters)
    finally:
        p.free()
        if exchange is None:
            x.free()
