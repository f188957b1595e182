"""Sharded batched paths (graphine_b200/shard.py) on the GPU: a one-rank NCCL group runs the same
code as N ranks (block split, batched kernels, one NCCL sum) and must give the unsharded results."""
import socket

import numpy as np
import pytest

import graphine_b200.gre as G
from graphine_b200 import shard

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nccl_group():
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(0)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    yield
    dist.destroy_process_group()


def test_sharded_bc_ppr_graph_batch_match_unsharded(nccl_group):
    n, off, col = G.rmat_host(14, 16, 8, True)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True, reorder=True)
    srcs = G.sample_sources(off, 130, 4)
    ref, _ = G.bc(g, srcs, batched=True)
    got = shard.bc(g, srcs)
    assert np.abs(got - ref).sum() <= 1e-12 * np.abs(ref).sum()
    lo, hi, rows = shard.ppr(g, srcs[:7])
    ref_rows, _ = G.ppr(g, srcs[:7])
    assert (lo, hi) == (0, 7)
    np.testing.assert_array_equal(rows, ref_rows.reshape(7, n))
    parts = [G.rmat_host(s, 16, 50 + s, True) for s in (9, 11, 10)]
    roots = [int(G.sample_sources(o, 1, 1)[0]) for _, o, _ in parts]
    lo, hi, lvs = shard.bfs_graph_batch(parts, roots)
    assert (lo, hi) == (0, 3)
    for (pn, po, pc), r, lv in zip(parts, roots, lvs):
        one = G.Graph.from_csr(pn, po, pc, dir=G.InOut, symmetric=True)
        ref_lv, _ = G.bfs(one, [r])
        np.testing.assert_array_equal(lv, ref_lv)
