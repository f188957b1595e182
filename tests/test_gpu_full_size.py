"""The benchmark's full-size workload (RMAT scale 26, edge factor 16, symmetric: 67.1M vertices,
2.10B arcs, relabelled) checked through size-independent properties, on the device (torch is only
the checker here; the oracle is too slow at this size):

* BFS: the root at level 0; the neighbours of a reached vertex are reached, one level apart at
  most; every other reached vertex has a neighbour one level up.
* SSSP (random uint32 weights in [1, 255]): no arc can shorten a distance; every reached
  non-root vertex has a tight arc (dist[u] + w == dist[v]).
* CC: labels constant along arcs, no larger than the vertex's id, the label's vertex labelled
  with itself, and a BFS from all self-labelled vertices reaching every vertex (so every label
  lies in its own component and is its smallest caller id).
* PageRank: superstep 21 recomputed from superstep 20 with an independent scatter-add in FP64
  (relative L1 difference <= 1e-12).
* The 1D-partitioned paths (two parts as threads on this GPU) equal the one-GPU results.
"""
import numpy as np
import pytest

import graphine_b200.gre as G
from graphine_b200 import partition as PT

pytestmark = pytest.mark.gpu
SCALE = 26
CHUNK = 1 << 28  # arcs per checked block (2 GB of int64 indices)


@pytest.fixture(scope="module")
def big():
    import torch

    g = G.Graph.rmat(SCALE, 16, 26, True, reorder=True)
    dev = torch.device("cuda", 0)
    off = torch.empty(g.n + 1, dtype=torch.int64, device=dev)
    col = torch.empty(g.m, dtype=torch.int32, device=dev)
    G._check(G.lib().gre_graph_csr(g._h, off.data_ptr(), col.data_ptr()), "gre_graph_csr")
    deg = off[1:] - off[:-1]
    yield g, off, col, deg
    g.free()
    torch.cuda.empty_cache()


def arc_blocks(off, col, deg):
    """(tail, head, first arc) per block of whole rows of at most CHUNK arcs (int64 tensors)."""
    import torch

    n = deg.numel()
    offh = off.cpu().numpy()
    r0 = 0
    while r0 < n:
        r1 = int(np.searchsorted(offh, offh[r0] + CHUNK, side="right")) - 1
        r1 = max(r1, r0 + 1)
        r1 = min(r1, n)
        a0, a1 = int(offh[r0]), int(offh[r1])
        tail = torch.repeat_interleave(torch.arange(r0, r1, device=off.device), deg[r0:r1])
        yield tail, col[a0:a1].long(), a0
        r0 = r1


def u32(t):
    return t.long() & 0xFFFFFFFF


def test_full_size_bfs_properties(big):
    import torch

    g, off, col, deg = big
    root = int(torch.nonzero(deg > 0)[5].item())
    lv = torch.empty(g.n, dtype=torch.int32, device=off.device)
    _, st = G.bfs(g, [root], out=lv)
    L = lv.long()
    assert int(L[root]) == 0 and st.traversed_edges > g.m // 4
    has_parent = torch.zeros(g.n, dtype=torch.bool, device=off.device)
    for tail, head, _ in arc_blocks(off, col, deg):
        a, b = L[tail], L[head]
        reached = a >= 0
        assert bool((b[reached] >= 0).all())
        assert bool(((a - b).abs()[reached] <= 1).all())
        has_parent[head[(b == a + 1) & reached]] = True
    assert bool(has_parent[L > 0].all())


def test_full_size_sssp_properties(big):
    import torch

    g, off, col, deg = big
    gen = torch.Generator(device=off.device).manual_seed(5)
    w = torch.randint(1, 256, (g.m,), dtype=torch.int32, device=off.device, generator=gen)
    g.loadEdgeProperty(w)  # caller CSR order, device buffer
    root = int(torch.nonzero(deg > 0)[17].item())
    dist = torch.empty(g.n, dtype=torch.int32, device=off.device)
    G.sssp(g, [root], out=dist)
    D = u32(dist)
    INF = 0xFFFFFFFF
    assert int(D[root]) == 0
    tight = torch.zeros(g.n, dtype=torch.bool, device=off.device)
    for tail, head, a0 in arc_blocks(off, col, deg):
        du, dv = D[tail], D[head]
        wt = w[a0:a0 + tail.numel()].long()
        fin = du != INF
        assert bool((dv[fin] <= du[fin] + wt[fin]).all())
        tight[head[fin & (dv == du + wt)]] = True
    reached = D != INF
    reached[root] = False
    assert bool(tight[reached].all())


def test_full_size_cc_properties(big):
    import torch

    g, off, col, deg = big
    lab = torch.empty(g.n, dtype=torch.int32, device=off.device)
    G.cc(g, out=lab)
    Lb = u32(lab)
    for tail, head, _ in arc_blocks(off, col, deg):
        assert bool((Lb[tail] == Lb[head]).all())
    ids = torch.arange(g.n, device=off.device)
    assert bool((Lb <= ids).all())
    assert bool((Lb[Lb] == Lb).all())
    # a BFS from every self-labelled vertex reaches all vertices: with labels constant along arcs,
    # each vertex's label then lies in its own component (two components cannot share a label)
    roots = torch.nonzero(Lb == ids).flatten().to(torch.int32)
    lv = torch.empty(g.n, dtype=torch.int32, device=off.device)
    G.bfs_multiroot(g, roots, out=lv)
    assert bool((lv >= 0).all())


def test_full_size_pagerank_superstep(big):
    import torch

    g, off, col, deg = big
    d = 0.85
    p20 = torch.empty(g.n, dtype=torch.float64, device=off.device)
    p21 = torch.empty_like(p20)
    G.pagerank(g, G.PR_ITER, d, 20, out=p20)
    G.pagerank(g, G.PR_ITER, d, 21, out=p21)
    contrib = torch.where(deg > 0, p20 / deg.clamp(min=1).double(), torch.zeros_like(p20))
    acc = torch.zeros_like(p20)
    for tail, head, _ in arc_blocks(off, col, deg):
        acc.index_add_(0, head, contrib[tail])
    expect = torch.where(deg > 0, (1 - d) + d * acc, torch.full_like(acc, 1 - d))  # symmetric: in-arcs = out-arcs
    rel = float((p21 - expect).abs().sum() / expect.abs().sum())
    assert rel <= 1e-12


def test_full_size_partitioned_equals_one_gpu(big):
    import torch

    g, off, col, deg = big
    root = int(torch.nonzero(deg > 0)[1000].item())
    g.set_weights_hash(7)
    one_lv, _ = G.bfs(g, [root])
    one_pr, _ = G.pagerank(g, G.PR_ITER, 0.85, 20)
    one_cc, _ = G.cc(g)
    one_d, _ = G.sssp(g, [root])
    # two parts: each part's rows still reach the CTA and hub-chunk bins of the degree schedule
    out = PT.run_local(g, 2, lambda part, x: (part.bfs(root, x)[0], part.pagerank(x, G.PR_ITER, 0.85, 20)[0],
                                              part.cc(x)[0], part.sssp(root, x)[0]))
    windows = g.row_schedule()[3] != 0  # source windows: a different association order per row
    for lv, pr, lab, dist in out:
        np.testing.assert_array_equal(lv, one_lv)
        if windows:
            assert np.abs(pr - one_pr).sum() <= 1e-12 * np.abs(one_pr).sum()
        else:
            np.testing.assert_array_equal(pr, one_pr)
        np.testing.assert_array_equal(lab, one_cc)
        np.testing.assert_array_equal(dist, one_d)
