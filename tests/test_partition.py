"""1D partition of one graph over ranks (graphine_b200/partition.py), on CPU.

The vertex layout (vertices dealt to ranks in snake order) is checked as a bijection onto the rank-major
exchange array, against the library's own host computation of it, and for balance of arcs on a
degree-ordered RMAT graph.  The torch.distributed exchange (the collectives the library calls
back into) is checked on gloo ranks with host buffers.  The partitioned kernels themselves are
in test_gpu_partition.py.
"""
import ctypes as C
import os
import socket
import subprocess
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

import graphine_b200.gre as G
from graphine_b200 import partition as PT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n", [1, 63, 64, 65, 1000, 4096 + 5, 3 * 64 * 7])
@pytest.mark.parametrize("P", [1, 2, 3, 8])
def test_layout_is_a_bijection_onto_rank_blocks(n, P):
    L, x = PT.layout(n, P)
    assert L % 64 == 0 and P * L >= n and L - (n + P - 1) // P < 64
    assert len(np.unique(x)) == n and x.min() >= 0 and x.max() < P * L
    rank, slot = x // L, x % L
    per_rank = np.bincount(rank, minlength=P)
    assert per_rank.max() - per_rank.min() <= 1
    for p in range(P):  # a rank's vertices fill its first slots, in increasing internal id
        ids = np.flatnonzero(rank == p)
        np.testing.assert_array_equal(slot[ids], np.arange(len(ids)))


@pytest.mark.parametrize("n,P", [(1, 1), (65, 3), (1000, 4), (4096 + 5, 8), (100000, 7)])
def test_library_layout_matches(n, P):
    L, x = PT.layout(n, P)
    L2, x2 = PT.library_layout(n, P)
    assert L == L2
    np.testing.assert_array_equal(x, x2)


def test_library_layout_rejects_zero_parts():
    L = C.c_uint64()
    assert G.lib().gre_part_layout(10, 0, C.byref(L), None) == G.GRE_INVALID_ARG


@pytest.mark.parametrize("P", [2, 4, 8])
def test_snake_order_balances_arcs_of_a_degree_ordered_graph(P):
    n, off, col = G.rmat_host(16, 16, 3, True)
    deg = np.sort(np.diff(off.astype(np.int64)))[::-1]  # internal ids by decreasing degree
    L, x = PT.layout(n, P)
    arcs = np.bincount(x // L, weights=deg, minlength=P)
    assert arcs.max() / arcs.mean() < 1.05  # rank 0 also holds the largest hub (0.5% of arcs here)


def test_nccl_communicator_arguments_checked_on_the_host():
    uid = (C.c_uint8 * 128)()
    assert G.lib().gre_nccl_create(None, 1, 0, 0, None) == G.GRE_NULL
    h = C.c_void_p()
    assert G.lib().gre_nccl_create(uid, 2, 2, 0, C.byref(h)) == G.GRE_INVALID_ARG
    assert G.lib().gre_nccl_create(uid, 0, 0, 0, C.byref(h)) == G.GRE_INVALID_ARG
    assert G.lib().gre_nccl_free(None) == G.GRE_SUCCESS
    # the exchange refuses a missing communicator instead of touching NCCL
    assert G.lib().gre_nccl_exchange(None, G.XCHG_ALLGATHER, None, None, 8, None) != 0
    # NCCL is opened on demand: an id comes back, or the status says NCCL is missing
    assert G.lib().gre_nccl_unique_id(uid) in (G.GRE_SUCCESS, G.GRE_NOT_IMPLEMENTED)


def _exchange_worker(rank, world, port, results):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        x = PT.TorchExchange(memory="host")
        nb = 24
        send = np.full(nb, rank + 1, dtype=np.uint8)
        recv = np.zeros(nb * world, dtype=np.uint8)
        x(PT.ALLGATHER, send.ctypes.data, recv.ctypes.data, nb, 0)
        gathered = recv.copy()
        send2 = (np.arange(nb * world) // nb * 16 + rank).astype(np.uint8)  # block q tagged (q, rank)
        recv2 = np.zeros(nb * world, dtype=np.uint8)
        x(PT.ALLTOALL, send2.ctypes.data, recv2.ctypes.data, nb, 0)
        results[rank] = (gathered, recv2.copy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_torch_exchange_semantics_over_gloo(world):
    ctx = mp.get_context("spawn")
    results = ctx.Manager().dict()
    mp.start_processes(_exchange_worker, args=(world, _free_port(), results), nprocs=world, join=True,
                       start_method="spawn")
    nb = 24
    for r in range(world):
        gathered, a2a = results[r]
        np.testing.assert_array_equal(gathered, np.repeat(np.arange(1, world + 1), nb))
        # block q of rank r's receive buffer = block r of rank q's send buffer
        np.testing.assert_array_equal(a2a, np.repeat(np.arange(world) + r * 16, nb))


DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "graphine_b200", "drivers", "gre_run")


def test_driver_partitioned_arguments_and_id_file():
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, "g")
        bad = subprocess.run([DRIVER, "part_bfs", prefix, "--ranks", "2", "--rank", "2", "--id-file", "x"],
                             capture_output=True, text=True, timeout=60)
        assert bad.returncode == 2
        bad = subprocess.run([DRIVER, "part_bfs", prefix, "--ranks", "1"], capture_output=True, text=True, timeout=60)
        assert bad.returncode == 2
        # rank 0 publishes the communicator id whole before it needs a GPU
        idf = os.path.join(td, "nccl.id")
        p = subprocess.run([DRIVER, "part_bfs", prefix, "--ranks", "1", "--rank", "0", "--id-file", idf],
                           capture_output=True, text=True, timeout=120)
        if G.device_count() == 0:
            assert p.returncode != 0
        assert os.path.getsize(idf) == 128 and not os.path.exists(idf + ".tmp")
