"""Degenerate inputs on every fast path and engine plugin, against the oracle restatement:
a graph without arcs, a single vertex, self loops and parallel arcs only, isolated sources,
sources repeated in one batch, a batch of exactly 64 / 65 sources (one full word and one bit
of the next), and a union with an empty member."""
import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O
from conftest import rel_l1

pytestmark = pytest.mark.gpu
TOL = 1e-9
REORDER = pytest.mark.parametrize("reorder", [False, True], ids=["plain", "relabelled"])


def csr(n, edges):
    src = np.array([e[0] for e in edges], dtype=np.int64)
    dst = np.array([e[1] for e in edges], dtype=np.uint32)
    order = np.argsort(src, kind="stable")
    off = np.zeros(n + 1, np.uint64)
    np.add.at(off, src + 1, 1)
    return np.cumsum(off).astype(np.uint64), dst[order]


def check_all(n, off, col, roots, reorder, wseed=5):
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True, reorder=reorder)
    g.set_weights_hash(wseed)
    R = O.Restatement.from_csr(n, off, col)
    roots = np.asarray(roots, np.uint32)
    pr_ref, _ = R.pagerank(1, 0.85, 20)
    assert rel_l1(G.pagerank(g, G.PR_ITER, 0.85, 20)[0], pr_ref) <= TOL
    assert rel_l1(G.vc_pagerank(g, G.PR_ITER, 20)[0], pr_ref) <= TOL
    lv_ref = R.bfs_many(roots)
    np.testing.assert_array_equal(G.bfs(g, roots)[0].reshape(len(roots), n), lv_ref)
    np.testing.assert_array_equal(G.msbfs(g, roots)[0].reshape(len(roots), n), lv_ref)
    np.testing.assert_array_equal(G.vc_bfs(g, int(roots[0]), G.In)[1], lv_ref[0])
    d_ref = R.sssp_many(roots, wseed)
    np.testing.assert_array_equal(G.sssp(g, roots)[0].reshape(len(roots), n), d_ref)
    np.testing.assert_array_equal(G.vc_sssp(g, int(roots[0]))[0], d_ref[0])
    lab_ref, _ = R.cc()
    np.testing.assert_array_equal(G.cc(g)[0], lab_ref)
    np.testing.assert_array_equal(G.vc_cc(g)[0], lab_ref)
    bc_ref, _ = R.bc(roots)
    b1, _ = G.bc(g, roots, batched=False)
    b2, _ = G.bc(g, roots, batched=True)
    np.testing.assert_array_equal(b1, b2)
    assert rel_l1(b1, bc_ref) <= TOL or np.abs(b1 - bc_ref).max() <= 1e-12
    ppr_ref = R.ppr(roots[:3], 0.85, 20)
    assert rel_l1(G.ppr(g, roots[:3], 0.85, 20)[0], ppr_ref.ravel()) <= TOL
    return g


@REORDER
def test_graph_without_arcs(reorder):
    n = 5
    off = np.zeros(n + 1, np.uint64)
    col = np.zeros(0, np.uint32)
    check_all(n, off, col, [0, 3], reorder)


@REORDER
def test_single_vertex_with_self_loop_and_parallel_arcs(reorder):
    check_all(1, *csr(1, [(0, 0), (0, 0)]), [0], reorder)


@REORDER
def test_isolated_sources_and_repeated_sources(reorder):
    n = 9
    edges = [(0, 1), (1, 0), (1, 2), (2, 1), (2, 2), (5, 6), (6, 5), (5, 6), (6, 5)]
    check_all(n, *csr(n, edges), [3, 0, 0, 8, 5], reorder)


@pytest.mark.parametrize("k", [64, 65])
def test_full_and_spilling_source_words(k):
    n, off, col = G.rmat_host(10, 8, 21, True)
    roots = G.sample_sources(off, k, 3)
    check_all(n, off, col, roots, True)


def test_union_with_an_empty_member():
    parts = [(3, *csr(3, [])), (4, *csr(4, [(0, 1), (1, 0), (2, 3), (3, 2)])), (1, *csr(1, []))]
    gs = [G.Graph.from_csr(n, o, c, dir=G.InOut, symmetric=True) for n, o, c in parts]
    u, voff = G.Graph.union(gs)
    assert list(voff) == [0, 3, 7, 8]
    lv, _ = G.bfs_multiroot(u, [1, 3 + 2, 7])
    np.testing.assert_array_equal(lv, [-1, 0, -1, -1, -1, 0, 1, 0])
    lab, _ = G.cc(u)
    np.testing.assert_array_equal(lab, [0, 1, 2, 3, 3, 5, 5, 7])


def test_zero_sources_and_zero_seeds():
    n, off, col = G.rmat_host(8, 8, 2, True)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True)
    b, _ = G.bc(g, np.zeros(0, np.uint32))
    assert not b.any()
    out, _ = G.ppr(g, np.zeros(0, np.uint32))
    assert out.size == 0


def test_graph_batch_run_equals_per_graph_calls():
    import torch

    scales = [9, 12, 7, 11, 10]
    gs, roots = [], []
    for i, s in enumerate(scales):
        n, off, col = G.rmat_host(s, 8, 40 + i, True)
        gs.append(G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True))
        roots.append(int(G.sample_sources(off, 1, i)[0]))
    dev_out = torch.empty(gs[1].n, dtype=torch.int32, device="cuda")
    outs = [np.empty(g.n, np.int32) for g in gs]
    outs[1] = dev_out
    lv, st = G.graph_batch_run(gs, G.BATCH_BFS, roots=roots, outs=outs)
    for g, r, x in zip(gs, roots, lv):
        got = x.cpu().numpy() if hasattr(x, "cpu") else x
        np.testing.assert_array_equal(got, G.bfs(g, [r])[0])
    assert st.supersteps > 0
    lab, _ = G.graph_batch_run(gs, G.BATCH_CC)
    for g, x in zip(gs, lab):
        np.testing.assert_array_equal(x, G.cc(g)[0])
    pr, _ = G.graph_batch_run(gs, G.BATCH_PAGERANK, variant=G.PR_ITER, d=0.85, iters=20)
    for g, x in zip(gs, pr):
        assert rel_l1(x, G.pagerank(g, G.PR_ITER, 0.85, 20)[0]) <= 1e-12
    with pytest.raises(G.GreError) as e:
        G.graph_batch_run(gs, G.BATCH_BFS, roots=[r + 10**6 for r in roots])
    assert e.value.status == G.GRE_INVALID_ARG
    with pytest.raises(G.GreError) as e:
        G.graph_batch_run(gs, 7)
    assert e.value.status == G.GRE_INVALID_ARG


@pytest.mark.parametrize("batched", [False, True], ids=["looped", "batched"])
def test_bc_on_a_long_path(batched):
    """A path of 6000 vertices: BFS levels run past 4096 from an end, and BC (looped and batched)
    equals the closed form (a source s adds to every v != s the number of vertices beyond v).

    The fast paths run BFS/BC to completion.  The reference engine stops every run after its
    default 1024 supersteps (Engine.hpp:108, which usr/test_bc.cpp does not raise), so on this
    graph its levels end at 1024; the device engine (gre_vc_*) keeps that limit, and the oracle
    restates it, which is why the closed form is the reference here."""
    n = 6000
    edges = [(i, i + 1) for i in range(n - 1)] + [(i + 1, i) for i in range(n - 1)]
    off, col = csr(n, edges)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True)
    roots = np.array([0, 2500, n - 1], np.uint32)
    v = np.arange(n, dtype=np.float64)
    ref = np.zeros(n)
    for s in roots:
        ref += np.where(v > s, n - 1 - v, np.where(v < s, v, 0.0))
    got, st = G.bc(g, roots, batched=batched)
    assert rel_l1(got, ref) <= TOL
    lv, _ = G.bfs(g, roots[:1])
    np.testing.assert_array_equal(lv, np.arange(n))
    R = O.Restatement.from_csr(n, off, col)  # the reference's engine limit, restated
    assert R.bfs(0)[0].max() == 1024


def test_device_inputs_ordered_after_the_default_stream():
    """A device buffer written on PyTorch's default stream just before the call (behind 0.1 s of
    queued GPU work) is read only after that write: the library's own stream is non-blocking, and
    each call orders it after the legacy default stream.  Weights loaded that way give the same
    distances as the same weights loaded from host memory; a device output that the default
    stream still reads is not overwritten early either."""
    import torch

    n, off, col = G.rmat_host(12, 16, 5, True)
    w_host = np.random.default_rng(1).integers(1, 256, size=len(col), dtype=np.uint32)
    ref_g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True)
    ref_g.loadEdgeProperty(w_host)
    roots = G.sample_sources(off, 2, 3)
    ref, _ = G.sssp(ref_g, roots)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True)
    g.loadEdgeProperty(np.ones(len(col), np.uint32))  # the weight array exists: no allocation orders the load below
    G.sssp(g, roots)  # and the run's scratch too
    staged = torch.from_numpy(w_host.view(np.int32)).cuda()
    torch.cuda.synchronize()
    torch.cuda._sleep(200_000_000)  # about 0.1 s of GPU time, then the copy the call must wait for
    w = staged.clone()
    g.loadEdgeProperty(w)
    got, _ = G.sssp(g, roots)
    np.testing.assert_array_equal(got, ref)
    out = torch.zeros(len(roots) * n, dtype=torch.int32, device="cuda")
    torch.cuda._sleep(200_000_000)
    before = out.clone()  # reads the zeros after the sleep: the call's writes must come later
    G.sssp(g, roots, out=out)
    torch.cuda.synchronize()
    assert int(before.abs().sum()) == 0
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), ref.reshape(-1))
