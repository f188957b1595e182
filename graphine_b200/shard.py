"""Batched units sharded over ranks: one process per GPU, no exchange during the run.

The reference runs many BC sources as a driver loop around one engine (usr/test_bc.cpp:63-110,
summing the per-source dependencies into one BC vector, BC.hpp:99-163) and spreads one graph over
MPI ranks.  Here the units of the batched paths are independent, so they are the thing that is
spread: BC sources and personalisation seeds are split into contiguous blocks of whole 64-source
words (a rank never splits a frontier word), every rank runs the batched kernels on its own GPU
with its own copy of the graph, and the only collective is one sum of the per-rank BC vectors
(8n bytes, NCCL on GPUs).  PPR rows and graph-batch members come back disjoint, with no
collective.

``torch.distributed`` is plumbing here: the process group, when one is initialised, decides the
rank and carries the sum.  Without one the functions run the whole batch on this process.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence, Tuple

import numpy as np

from . import gre as G

WORD = 64  # sources per frontier word of the batched BC / BFS


def _rank_world(group=None) -> Tuple[int, int]:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def shard_range(k: int, rank: int, world: int, align: int = WORD) -> Tuple[int, int]:
    """Half-open block [lo, hi) of k units for `rank`: blocks of whole `align`-unit groups, group
    counts differing by at most one between ranks, in rank order (so the blocks tile [0, k))."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    groups = (k + align - 1) // align
    base, extra = divmod(groups, world)
    g0 = rank * base + min(rank, extra)
    g1 = g0 + base + (1 if rank < extra else 0)
    return min(k, g0 * align), min(k, g1 * align)


def _sum_over_ranks(x: np.ndarray, group=None) -> np.ndarray:
    """Element-wise sum over the ranks of the group (NCCL for CUDA tensors, gloo for host)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return x
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def bc(g: "G.Graph", srcs: Sequence[int], group=None,
       partial: Optional[Callable[[np.ndarray], np.ndarray]] = None) -> np.ndarray:
    """Betweenness over all `srcs`, the sources spread over the ranks of `group`.

    Every rank returns the full BC vector (the sum of the ranks' partial vectors).  `partial`
    computes one rank's vector from its block of sources; it defaults to the batched GPU path
    (`gre_bc`, 64 sources per word) on this rank's graph handle."""
    s = np.ascontiguousarray(srcs, dtype=np.uint32)
    rank, world = _rank_world(group)
    lo, hi = shard_range(len(s), rank, world)
    if partial is None:
        partial = lambda block: G.bc(g, block, batched=True)[0]  # noqa: E731
    local = partial(s[lo:hi]) if hi > lo else np.zeros(g.n if g is not None else 0, dtype=np.float64)
    return _sum_over_ranks(np.asarray(local, dtype=np.float64), group)


def ppr(g: "G.Graph", seeds: Sequence[int], d: float = 0.85, iters: int = 20, group=None,
        partial: Optional[Callable[[np.ndarray], np.ndarray]] = None) -> Tuple[int, int, np.ndarray]:
    """Personalised PageRank rows for this rank's block of `seeds`: returns (lo, hi, rows) with
    rows[i] the vector of seeds[lo + i].  No collective: the blocks are disjoint."""
    s = np.ascontiguousarray(seeds, dtype=np.uint32)
    rank, world = _rank_world(group)
    lo, hi = shard_range(len(s), rank, world, align=1)
    if partial is None:
        partial = lambda block: G.ppr(g, block, d, iters, batched=True)[0]  # noqa: E731
    n = g.n if g is not None else 0
    rows = np.asarray(partial(s[lo:hi]), dtype=np.float64).reshape(hi - lo, -1) if hi > lo else np.zeros((0, n))
    return lo, hi, rows


def bfs_graph_batch(parts: Sequence[Tuple[int, np.ndarray, np.ndarray]], roots: Sequence[int], group=None,
                    device: int = 0) -> Tuple[int, int, list]:
    """BFS levels for this rank's block of a batch of graphs (n, off, col) with one root each:
    the block is joined into one block-diagonal graph and run as one multi-root BFS.  Returns
    (lo, hi, levels) with levels[i] the levels of graph lo + i."""
    rank, world = _rank_world(group)
    lo, hi = shard_range(len(parts), rank, world, align=1)
    if hi == lo:
        return lo, hi, []
    gs = [G.Graph.from_csr(n, o, c, dir=G.InOut, symmetric=True, device=device) for n, o, c in parts[lo:hi]]
    u, voff = G.Graph.union(gs, device=device)
    lv, _ = G.bfs_multiroot(u, [int(r) + int(voff[i]) for i, r in enumerate(roots[lo:hi])])
    return lo, hi, [lv[int(voff[i]):int(voff[i + 1])] for i in range(hi - lo)]
