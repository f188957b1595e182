"""1D-partitioned single-source paths (gre_part_*) on the GPU.

P parts of one graph run as P threads of this process on one GPU, their collectives meeting at
a host barrier (partition.LocalExchange: no kernel waits for another); the NCCL exchange runs
as a one-rank process group.  Levels must equal the oracle's and the one-GPU path's bit for bit;
PageRank must equal the one-GPU path bit for bit (same row schedule, same association order) and
the oracle within 1e-9.
"""
import socket

import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O
from conftest import rel_l1
from graphine_b200 import partition as PT

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _graph(scale, symmetric, reorder, seed=7):
    n, off, col = G.rmat_host(scale, 8, seed, symmetric)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut if symmetric else G.Out, symmetric=symmetric, reorder=reorder)
    return n, off, col, g


@pytest.mark.parametrize("P", [1, 2, 3, 4])
@pytest.mark.parametrize("reorder", [False, True], ids=["plain", "relabelled"])
def test_partitioned_bfs_equals_oracle_and_one_gpu(P, reorder):
    n, off, col, g = _graph(11, True, reorder)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 3, 4)
    ref = R.bfs_many(roots)
    for i, s in enumerate(roots):
        one, st1 = G.bfs(g, [s])
        out = PT.run_local(g, P, lambda part, x: part.bfs(int(s), x))
        for lv, st in out:
            np.testing.assert_array_equal(lv, ref[i])
            np.testing.assert_array_equal(lv, one)
            assert st.supersteps == st1.supersteps
            assert st.active == st1.active
            assert st.traversed_edges == st1.traversed_edges


@pytest.mark.parametrize("P", [1, 2, 3, 4])
@pytest.mark.parametrize("variant", [G.PR_REFERENCE, G.PR_ITER], ids=["reference", "iter"])
def test_partitioned_pagerank_equals_one_gpu_bitwise(P, variant):
    n, off, col, g = _graph(11, True, True)
    one, _ = G.pagerank(g, variant, 0.85, 20)
    R = O.Restatement.from_csr(n, off, col)
    ref, _ = R.pagerank(variant, 0.85, 20)
    out = PT.run_local(g, P, lambda part, x: part.pagerank(x, variant, 0.85, 20))
    for pr, st in out:
        np.testing.assert_array_equal(pr, one)
        assert rel_l1(pr, ref) <= TOL
        assert st.supersteps == 20


@pytest.mark.parametrize("P", [2, 3])
def test_partitioned_directed_graph(P):
    n, off, col, g = _graph(10, False, True, seed=3)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 2, 9)
    ref = R.bfs_many(roots, G.Out)  # levels along out-arcs, as gre_bfs
    for i, s in enumerate(roots):
        one, _ = G.bfs(g, [s])
        np.testing.assert_array_equal(one, ref[i])
        for lv, _ in PT.run_local(g, P, lambda part, x: part.bfs(int(s), x)):
            np.testing.assert_array_equal(lv, ref[i])
    one, _ = G.pagerank(g, G.PR_ITER, 0.85, 20)
    for pr, _ in PT.run_local(g, P, lambda part, x: part.pagerank(x, G.PR_ITER, 0.85, 20)):
        np.testing.assert_array_equal(pr, one)


WSEED = 11


@pytest.mark.parametrize("P", [1, 2, 3, 4])
@pytest.mark.parametrize("reorder", [False, True], ids=["plain", "relabelled"])
def test_partitioned_sssp_equals_oracle_and_one_gpu(P, reorder):
    n, off, col, g = _graph(11, True, reorder)
    g.set_weights_hash(WSEED)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 2, 5)
    ref = R.sssp_many(roots, WSEED)
    for i, s in enumerate(roots):
        one, st1 = G.sssp(g, [s])
        np.testing.assert_array_equal(one, ref[i])
        for dist, st in PT.run_local(g, P, lambda part, x: part.sssp(int(s), x)):
            np.testing.assert_array_equal(dist, ref[i])
            assert st.traversed_edges == st1.traversed_edges


@pytest.mark.parametrize("sparse", ["0", "1"], ids=["dense", "lists"])
@pytest.mark.parametrize("pull", ["0", "1"], ids=["push", "pull"])
@pytest.mark.parametrize("binned", ["0", "4294967296"], ids=["tiles", "bins"])
@pytest.mark.parametrize("P", [1, 3])
def test_partitioned_sssp_forms(monkeypatch, P, binned, pull, sparse):
    """Every relaxation form of the partitioned SSSP (arc tiles or the rank's degree bins for the
    light offers and the pushed heavy offers, or the pulled heavy pass; light offers exchanged as
    dense per-owner arrays, or as (slot, distance) lists whenever they fit half the dense bytes)
    on a schedule whose short CTA threshold and hub chunks put rows into the CTA and chunk bins
    of each part."""
    monkeypatch.setenv("GRE_ROW_SCHEDULE", "2,32,64,0")
    monkeypatch.setenv("GRE_SSSP_BINNED", binned)
    monkeypatch.setenv("GRE_SSSP_PULL", pull)
    monkeypatch.setenv("GRE_PART_SPARSE", sparse)
    n, off, col, g = _graph(11, True, True)
    g.set_weights_hash(WSEED)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 2, 6)
    ref = R.sssp_many(roots, WSEED)
    for i, s in enumerate(roots):
        for dist, _ in PT.run_local(g, P, lambda part, x: part.sssp(int(s), x)):
            np.testing.assert_array_equal(dist, ref[i])


@pytest.mark.parametrize("pull_arcs", ["0", "4294967296"], ids=["by-members", "heavy-always"])
@pytest.mark.parametrize("P", [1, 3])
def test_partitioned_sssp_heavy_pull_by_arcs(monkeypatch, P, pull_arcs):
    """Heavy passes pulled by the bucket's member count only, or whenever it has any heavy arcs
    (the decision from the all-gathered sums, the same on every rank)."""
    monkeypatch.setenv("GRE_SSSP_PULL_ARCS", pull_arcs)
    n, off, col, g = _graph(11, True, True)
    g.set_weights_hash(WSEED)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 2, 8)
    ref = R.sssp_many(roots, WSEED)
    for i, s in enumerate(roots):
        for dist, _ in PT.run_local(g, P, lambda part, x: part.sssp(int(s), x)):
            np.testing.assert_array_equal(dist, ref[i])


@pytest.mark.parametrize("P", [1, 2, 3, 4])
@pytest.mark.parametrize("reorder", [False, True], ids=["plain", "relabelled"])
def test_partitioned_cc_equals_oracle_and_one_gpu(P, reorder):
    n, off, col, g = _graph(11, True, reorder)
    R = O.Restatement.from_csr(n, off, col)
    ref, _ = R.cc()
    one, _ = G.cc(g)
    np.testing.assert_array_equal(one, ref)
    assert len(np.unique(ref)) > 1  # several components (isolated vertices among them)
    for lab, st in PT.run_local(g, P, lambda part, x: part.cc(x)):
        np.testing.assert_array_equal(lab, ref)
        assert st.active[-1] == 0


@pytest.mark.parametrize("P", [2, 3])
def test_partitioned_sssp_and_cc_directed(P):
    n, off, col, g = _graph(10, False, True, seed=3)
    g.set_weights_hash(WSEED)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 2, 9)
    ref = R.sssp_many(roots, WSEED)
    for i, s in enumerate(roots):
        for dist, _ in PT.run_local(g, P, lambda part, x: part.sssp(int(s), x)):
            np.testing.assert_array_equal(dist, ref[i])
    one, _ = G.cc(g)  # weak components
    for lab, _ in PT.run_local(g, P, lambda part, x: part.cc(x)):
        np.testing.assert_array_equal(lab, one)


def test_partitioned_sssp_needs_weights_at_creation():
    n, off, col, g = _graph(9, True, False)
    p = PT.Part(g, 1, 0)
    g.set_weights_hash(WSEED)  # too late for this part
    with pytest.raises(G.GreError) as e:
        p.sssp(0, PT.LocalExchange(1).for_rank(0))
    assert e.value.status == G.GRE_INVALID_ARG
    p.free()
    p = PT.Part(g, 1, 0)
    dist, _ = p.sssp(0, PT.LocalExchange(1).for_rank(0))
    np.testing.assert_array_equal(dist, G.sssp(g, [0])[0])
    p.free()


def test_parts_with_only_padding_and_isolated_source():
    # 5 vertices over 4 ranks: rank slots of 64, most of them padding
    n = 5
    src = np.array([0, 1, 1, 2, 3, 4], dtype=np.int64)
    dst = np.array([1, 0, 2, 1, 4, 3], dtype=np.uint32)
    order = np.argsort(src, kind="stable")
    off = np.zeros(n + 1, np.uint64)
    np.add.at(off, src + 1, 1)
    off = np.cumsum(off).astype(np.uint64)
    col = dst[order]
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True)
    for part_out in PT.run_local(g, 4, lambda part, x: (part.slots, part.bfs(0, x)[0], part.bfs(3, x)[0])):
        slots, a, b = part_out
        assert slots == 64
        np.testing.assert_array_equal(a, [0, 1, 2, -1, -1])
        np.testing.assert_array_equal(b, [-1, -1, -1, 0, 1])
    empty = G.Graph.from_csr(3, np.zeros(4, np.uint64), np.zeros(0, np.uint32), dir=G.InOut, symmetric=True)
    for lv, st in PT.run_local(empty, 2, lambda part, x: part.bfs(1, x)):
        np.testing.assert_array_equal(lv, [-1, 0, -1])
        assert st.supersteps == 0
    one, _ = G.pagerank(empty, G.PR_ITER, 0.85, 5)
    for pr, _ in PT.run_local(empty, 2, lambda part, x: part.pagerank(x, G.PR_ITER, 0.85, 5)):
        np.testing.assert_array_equal(pr, one)


def test_errors_are_statuses_and_the_part_stays_usable():
    n, off, col, g = _graph(9, True, False)
    p = PT.Part(g, 1, 0)
    x = PT.LocalExchange(1).for_rank(0)
    with pytest.raises(G.GreError) as e:
        p.bfs(n, x)
    assert e.value.status == G.GRE_INVALID_ARG
    calls = []

    def failing(kind, s, r, nb, st):
        calls.append(kind)
        if len(calls) == 3:
            raise RuntimeError("peer left")
        x(kind, s, r, nb, st)

    with pytest.raises(G.GreError) as e:
        p.bfs(0, failing)
    assert e.value.status == G.GRE_FAILURE and "peer left" in str(e.value)
    lv, _ = p.bfs(0, x)
    np.testing.assert_array_equal(lv, G.bfs(g, [0])[0])
    with pytest.raises(G.GreError) as e:
        PT.Part(g, 2, 2)
    assert e.value.status == G.GRE_INVALID_ARG
    p.free()


def test_part_outlives_its_graph():
    n, off, col, g = _graph(10, True, True)
    one, _ = G.bfs(g, [5])
    parts = [PT.Part(g, 2, r) for r in range(2)]
    g.free()
    x = PT.LocalExchange(2)
    import threading

    res = [None, None]

    def work(r):
        res[r] = parts[r].bfs(5, x.for_rank(r))[0]

    ts = [threading.Thread(target=work, args=(r,)) for r in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for r in range(2):
        np.testing.assert_array_equal(res[r], one)
        parts[r].free()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_nccl_exchange_one_rank_group():
    import torch
    import torch.distributed as dist

    n, off, col, g = _graph(12, True, True)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        lv, _ = PT.bfs(g, 17, exchange=PT.TorchExchange())
        np.testing.assert_array_equal(lv, G.bfs(g, [17])[0])
        pr, _ = PT.pagerank(g, G.PR_ITER, 0.85, 20, exchange=PT.TorchExchange())
        np.testing.assert_array_equal(pr, G.pagerank(g, G.PR_ITER, 0.85, 20)[0])
        lv, _ = PT.bfs(g, 17)  # the library's communicator, id carried by the group
        np.testing.assert_array_equal(lv, G.bfs(g, [17])[0])
        # device outputs through the same exchange
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        p = PT.Part(g, 1, 0)
        p.pagerank(PT.TorchExchange(), G.PR_REFERENCE, 0.85, 10, out=out)
        np.testing.assert_array_equal(out.cpu().numpy(), G.pagerank(g, G.PR_REFERENCE, 0.85, 10)[0])
        p.free()
    finally:
        dist.destroy_process_group()


def test_library_nccl_exchange_one_rank():
    import torch

    n, off, col, g = _graph(12, True, True)
    g.set_weights_hash(WSEED)
    x = PT.NcclExchange()
    p = PT.Part(g, 1, 0)
    try:
        for src in (0, 17, 1000):
            lv, st = p.bfs(src, x)
            one, st1 = G.bfs(g, [src])
            np.testing.assert_array_equal(lv, one)
            assert st.active == st1.active
        for variant in (G.PR_REFERENCE, G.PR_ITER):
            out = torch.empty(n, dtype=torch.float64, device="cuda")
            p.pagerank(x, variant, 0.85, 20, out=out)
            np.testing.assert_array_equal(out.cpu().numpy(), G.pagerank(g, variant, 0.85, 20)[0])
        np.testing.assert_array_equal(p.cc(x)[0], G.cc(g)[0])
        np.testing.assert_array_equal(p.sssp(17, x)[0], G.sssp(g, [17])[0])
    finally:
        p.free()
        x.free()


def test_torch_exchange_stages_device_buffers_through_gloo():
    import torch.distributed as dist

    n, off, col, g = _graph(11, True, True)
    g.set_weights_hash(WSEED)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1)
    try:
        x = PT.TorchExchange()  # device buffers, host staging (gloo has no device collectives here)
        p = PT.Part(g, 1, 0)
        np.testing.assert_array_equal(p.bfs(3, x)[0], G.bfs(g, [3])[0])
        np.testing.assert_array_equal(p.sssp(3, x)[0], G.sssp(g, [3])[0])
        np.testing.assert_array_equal(p.pagerank(x, G.PR_ITER, 0.85, 10)[0], G.pagerank(g, G.PR_ITER, 0.85, 10)[0])
        p.free()
    finally:
        dist.destroy_process_group()
