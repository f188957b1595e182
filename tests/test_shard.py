"""Sharded batched paths over ranks (graphine_b200/shard.py), on CPU with gloo.

The per-rank computation is the oracle's restatement here (these tests check the split of the
units, the one sum of BC vectors and the disjoint PPR blocks, not the kernels); the GPU path
of the same functions is checked in test_gpu_shard.py.
"""
import os
import socket
import sys
import types

import numpy as np
import pytest
import torch.multiprocessing as mp

import graphine_b200.gre as G
from graphine_b200 import shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("k", [0, 1, 63, 64, 65, 200, 256, 1024, 1000])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_range_tiles_in_whole_words(k, world):
    blocks = [shard.shard_range(k, r, world) for r in range(world)]
    assert blocks[0][0] == 0 and blocks[-1][1] == k
    for (a0, a1), (b0, b1) in zip(blocks, blocks[1:]):
        assert a1 == b0  # contiguous, in rank order
    words = [((hi - lo) + 63) // 64 for lo, hi in blocks]
    assert max(words) - min(words) <= 1
    for lo, hi in blocks:
        assert (lo % 64 == 0 or lo == k) and (hi % 64 == 0 or hi == k)  # an empty block may sit at k


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, scale, nsrc, results):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))  # spawned: conftest's path setup is not inherited
    import torch.distributed as dist

    import oracle as O

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        n, off, col = G.rmat_host(scale, 16, 31, True)
        R = O.Restatement.from_csr(n, off, col)
        srcs = G.sample_sources(off, nsrc, 2)
        g = types.SimpleNamespace(n=n)
        bc = shard.bc(g, srcs, partial=lambda block: R.bc(block)[0])
        lo, hi, rows = shard.ppr(g, srcs[:10], partial=lambda block: R.ppr(block, 0.85, 20))
        results[rank] = (bc, lo, hi, rows)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_bc_and_ppr_sharded_over_gloo_ranks(world):
    import oracle as O

    scale, nsrc = 10, 150
    ctx = mp.get_context("spawn")
    results = ctx.Manager().dict()
    mp.start_processes(_worker, args=(world, _free_port(), scale, nsrc, results), nprocs=world, join=True,
                       start_method="spawn")
    n, off, col = G.rmat_host(scale, 16, 31, True)
    R = O.Restatement.from_csr(n, off, col)
    srcs = G.sample_sources(off, nsrc, 2)
    ref, _ = R.bc(srcs)
    for r in range(world):
        bc = results[r][0]
        assert np.abs(bc - ref).sum() <= 1e-12 * np.abs(ref).sum()  # every rank holds the full sum
    covered = sorted((results[r][1], results[r][2]) for r in range(world))
    assert covered[0][0] == 0 and covered[-1][1] == 10
    full = R.ppr(srcs[:10], 0.85, 20)
    for r in range(world):
        lo, hi, rows = results[r][1:]
        np.testing.assert_array_equal(rows, full[lo:hi])
