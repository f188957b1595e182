"""GPU parity: every entry point of libgre_gpu.so against the oracle.

* golden fixtures (outputs of the reference GRE engine, tests/golden/): bit-exact for BFS levels,
  SSSP distances, CC labels and per-superstep active counts; FP64 results within 1e-9 relative L1;
* seeded RMAT graphs up to scale 16 against the C++ restatement (oracle/gre_oracle.cpp);
* scale-20 graphs through size-independent properties (BFS level consistency, SSSP
  tightness, CC closure) that the oracle cannot afford at that size in a test.
"""
import os
import tempfile

import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O
from conftest import golden_cases, rel_l1

pytestmark = pytest.mark.gpu

TOL = 1e-9  # FP64 relative L1
CASES = golden_cases()
SYM = [c for c in CASES if not c.endswith("dir")]


def graph_of(case, reorder=False):
    sym = bool(case["symmetric"])
    return G.Graph.from_csr(int(case["n"]), case["off"], case["col"], dir=G.InOut if sym else G.Out, symmetric=sym,
                            reorder=reorder)


REORDER = pytest.mark.parametrize("reorder", [False, True], ids=["plain", "relabelled"])


# ---------------------------------------------------------------------------------------------
# golden fixtures (reference outputs)
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", CASES)
@REORDER
def test_pagerank_golden(golden, name, reorder):
    case = golden[name]
    g = graph_of(case, reorder)
    pr, st = G.vc_pagerank(g, G.PR_REFERENCE, 10)
    assert rel_l1(pr, case["pr_gre10"]) <= TOL
    assert st.supersteps == 10 and st.active == list(case["pr_gre10_active"])
    pr, st = G.vc_pagerank(g, G.PR_ITER, 20)
    assert rel_l1(pr, case["pr_iter20"]) <= TOL
    assert st.active == list(case["pr_iter20_active"])
    pr, _ = G.pagerank(g, G.PR_REFERENCE, 0.85, 10)
    assert rel_l1(pr, case["pr_gre10"]) <= TOL
    pr, _ = G.pagerank(g, G.PR_ITER, 0.85, 20)
    assert rel_l1(pr, case["pr_iter20"]) <= TOL


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("batched", [False, True])
@REORDER
def test_ppr_golden(golden, name, batched, reorder):
    case = golden[name]
    g = graph_of(case, reorder)
    out, _ = G.ppr(g, case["roots"][:2], 0.85, 20, batched=batched)
    assert rel_l1(out, case["ppr20"].ravel()) <= TOL


@pytest.mark.parametrize("name", SYM)
@REORDER
def test_bfs_golden(golden, name, reorder):
    case = golden[name]
    g = graph_of(case, reorder)
    roots = case["roots"]
    for i, r in enumerate(roots):
        pred, level, st = G.vc_bfs(g, int(r), G.In)
        np.testing.assert_array_equal(level, case["bfs_level"][i])
        assert st.active == [x for x in case["bfs_active"][i] if x >= 0]
        assert np.all((pred == int(r)) == (level >= 0))
        lv, st = G.bfs(g, [r])
        np.testing.assert_array_equal(lv, case["bfs_level"][i])
        assert st.active == [x for x in case["bfs_active"][i] if x >= 0]
    lv, _ = G.msbfs(g, roots)
    np.testing.assert_array_equal(lv.reshape(len(roots), -1), case["bfs_level"])
    lv, _ = G.bfs(g, roots)
    np.testing.assert_array_equal(lv.reshape(len(roots), -1), case["bfs_level"])


@pytest.mark.parametrize("name", SYM)
@REORDER
def test_sssp_golden(golden, name, reorder):
    case = golden[name]
    g = graph_of(case, reorder)
    g.set_weights_hash(int(case["wseed"]))
    for i, r in enumerate(case["roots"]):
        dist, st, status = G.vc_sssp(g, int(r))
        assert status == G.GRE_SUCCESS
        np.testing.assert_array_equal(dist, case["sssp_dist"][i])
        assert st.active == [x for x in case["sssp_active"][i] if x >= 0]
    dist, _ = G.sssp(g, case["roots"])
    np.testing.assert_array_equal(dist.reshape(len(case["roots"]), -1), case["sssp_dist"])


@pytest.mark.parametrize("name", SYM)
@REORDER
def test_cc_golden(golden, name, reorder):
    case = golden[name]
    g = graph_of(case, reorder)
    lab, st = G.vc_cc(g)
    np.testing.assert_array_equal(lab, case["cc_label"])
    assert st.active == list(case["cc_active"])
    lab, _ = G.cc(g)
    np.testing.assert_array_equal(lab, case["cc_label"])


@pytest.mark.parametrize("name", SYM)
@REORDER
def test_bc_golden(golden, name, reorder):
    case = golden[name]
    g = graph_of(case, reorder)
    b, _ = G.vc_bc(g, case["roots"])
    assert rel_l1(b, case["bc"]) <= TOL
    b1, _ = G.bc(g, case["roots"], batched=False)
    b2, _ = G.bc(g, case["roots"], batched=True)
    assert rel_l1(b1, case["bc"]) <= TOL
    np.testing.assert_array_equal(b1, b2)  # batched and looped: identical bits


@pytest.mark.parametrize("name", CASES)
@REORDER
def test_pagerank_delta_golden(golden, name, reorder):
    case = golden[name]
    g = graph_of(case, reorder)
    pr, st, status = G.vc_pagerank_delta(g)
    assert status == G.GRE_SUCCESS
    assert rel_l1(pr, case["prdelta"]) <= TOL
    assert st.active == list(case["prdelta_active"])


@pytest.mark.parametrize("name", SYM)
@REORDER
def test_sssp1_golden(golden, name, reorder):
    from test_oracle_golden import pred_tree_ok

    case = golden[name]
    g = graph_of(case, reorder)
    wseed = int(case["wseed"])
    g.set_weights_hash(wseed)
    for i, r in enumerate(case["roots"]):
        dist, pred, st, status = G.vc_sssp1(g, int(r))
        assert status == G.GRE_SUCCESS
        np.testing.assert_array_equal(dist, case["sssp1_dist"][i])
        assert st.active == [x for x in case["sssp1_active"][i] if x >= 0]
        assert pred_tree_ok(case["off"], case["col"], wseed, int(r), dist, pred)


@pytest.mark.parametrize("name", SYM)
@REORDER
def test_count_in_golden(golden, name, reorder):
    case = golden[name]
    g = graph_of(case, reorder)
    cn, st = G.vc_count_in(g, G.In, 1)
    np.testing.assert_array_equal(cn, case["countin"])
    assert st.active == list(case["countin_active"])


@pytest.mark.parametrize("name", CASES)
def test_loader_matches_fixture(golden, name):
    """gre_graph_load on the text files gives the fixture's CSR (file order within a source)."""
    case = golden[name]
    if name.startswith("toy"):
        pytest.skip("hand-written text; covered by the oracle tests")
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        G.write_edgelists(p, int(case["n"]), case["off"], case["col"], 4)
        g = G.Graph.ingress(p, G.InOut)
    off, col = g.csr()
    np.testing.assert_array_equal(off, case["off"])
    np.testing.assert_array_equal(col, case["col"])
    np.testing.assert_array_equal(g.getOutdegree(), np.diff(case["off"].astype(np.int64)))


# ---------------------------------------------------------------------------------------------
# seeded RMAT vs the restatement
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module", params=[False, True], ids=["plain", "relabelled"])
def rmat14(request):
    n, off, col = G.rmat_host(14, 16, 42, True)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True, reorder=request.param)
    if request.param:
        o2, c2 = g.csr()  # caller ids and caller arc order survive the relabelling
        np.testing.assert_array_equal(o2, off)
        np.testing.assert_array_equal(c2, col)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 16, 9)
    return n, off, col, g, R, roots


def test_rmat14_device_generator_matches_host():
    n, off, col = G.rmat_host(14, 16, 42, True)
    g = G.Graph.rmat(14, 16, 42, True)
    o2, c2 = g.csr()
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(c2, col)
    n, off, col = G.rmat_host(13, 8, 5, False)
    g = G.Graph.rmat(13, 8, 5, False)
    o2, c2 = g.csr()
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(c2, col)


def test_rmat14_bfs(rmat14):
    n, off, col, g, R, roots = rmat14
    ref = R.bfs_many(roots)
    lv, st = G.bfs(g, roots)
    np.testing.assert_array_equal(lv.reshape(len(roots), n), ref)
    lv, _ = G.msbfs(g, roots)
    np.testing.assert_array_equal(lv.reshape(len(roots), n), ref)
    assert st.traversed_edges > 0


def test_rmat14_sssp(rmat14):
    n, off, col, g, R, roots = rmat14
    g.set_weights_hash(77)
    ref = R.sssp_many(roots, 77)
    d, _ = G.sssp(g, roots)
    np.testing.assert_array_equal(d.reshape(len(roots), n), ref)
    d0, _, _ = G.vc_sssp(g, int(roots[0]))
    np.testing.assert_array_equal(d0, ref[0])


@pytest.mark.parametrize("delta", [0, 1, 7, 64, 1000])
def test_rmat14_sssp_near_far(rmat14, monkeypatch, delta):
    """Every near-far bucket width gives the oracle's distances (0 = Bellman-Ford frontier)."""
    n, off, col, g, R, roots = rmat14
    g.set_weights_hash(78)
    ref = R.sssp_many(roots, 78)
    monkeypatch.setenv("GRE_SSSP_DELTA", str(delta))
    d, st = G.sssp(g, roots)
    np.testing.assert_array_equal(d.reshape(len(roots), n), ref)


def test_rmat14_cc(rmat14):
    n, off, col, g, R, roots = rmat14
    ref, _ = R.cc()
    lab, _ = G.cc(g)
    np.testing.assert_array_equal(lab, ref)
    lab, _ = G.vc_cc(g)
    np.testing.assert_array_equal(lab, ref)


def test_rmat14_pagerank(rmat14):
    n, off, col, g, R, roots = rmat14
    for variant, ss in [(0, 10), (1, 20)]:
        ref, _ = R.pagerank(variant, 0.85, ss)
        pr, _ = G.pagerank(g, variant, 0.85, ss)
        assert rel_l1(pr, ref) <= TOL
        pr, _ = G.vc_pagerank(g, variant, ss)
        assert rel_l1(pr, ref) <= TOL


def test_rmat14_bc_batched_equals_looped(rmat14):
    n, off, col, g, R, roots = rmat14
    srcs = G.sample_sources(off, 70, 3)  # more than one 64-source word
    ref, ovf = R.bc(srcs)
    b1, _ = G.bc(g, srcs, batched=False)
    b2, _ = G.bc(g, srcs, batched=True)
    np.testing.assert_array_equal(b1, b2)
    assert rel_l1(b2, ref) <= TOL


def test_rmat14_ppr(rmat14):
    n, off, col, g, R, roots = rmat14
    seeds = roots[:5]
    ref = R.ppr(seeds, 0.85, 20)
    a, _ = G.ppr(g, seeds, 0.85, 20, batched=True)
    b, _ = G.ppr(g, seeds, 0.85, 20, batched=False)
    assert rel_l1(a, ref.ravel()) <= TOL
    assert rel_l1(b, ref.ravel()) <= TOL


def test_directed_pagerank_s16():
    n, off, col = G.rmat_host(16, 16, 1, False)
    g = G.Graph.from_csr(n, off, col, dir=G.Out)
    R = O.Restatement.from_csr(n, off, col)
    for variant, ss in [(0, 20), (1, 20)]:
        ref, _ = R.pagerank(variant, 0.85, ss)
        pr, st = G.pagerank(g, variant, 0.85, ss)
        assert rel_l1(pr, ref) <= TOL
        assert st.traversed_edges == g.m * ss


# ---------------------------------------------------------------------------------------------
# device buffers, errors
# ---------------------------------------------------------------------------------------------
def test_device_buffers_roundtrip(rmat14):
    import torch

    n, off, col, g, R, roots = rmat14
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    G.bfs(g, torch.tensor(roots[:1].astype(np.int32), device="cuda"), out=out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), R.bfs(int(roots[0]))[0])
    pr = torch.empty(n, dtype=torch.float64, device="cuda")
    G.pagerank(g, G.PR_ITER, 0.85, 20, out=pr)
    torch.cuda.synchronize()
    ref, _ = R.pagerank(1, 0.85, 20)
    assert rel_l1(pr.cpu().numpy(), ref) <= TOL


def test_errors_are_status_codes(rmat14):
    n, off, col, g, R, roots = rmat14
    with pytest.raises(G.GreError) as e:
        G.bfs(g, [n + 5])
    assert e.value.status == G.GRE_INVALID_ARG
    g2 = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True)
    with pytest.raises(G.GreError) as e:
        G.sssp(g2, [0])  # no weights
    assert e.value.status == G.GRE_INVALID_ARG
    with pytest.raises(G.GreError) as e:
        G.pagerank(g2, 7)
    assert e.value.status == G.GRE_INVALID_ARG


# ---------------------------------------------------------------------------------------------
# batch of uneven graphs in one launch (block-diagonal union)
# ---------------------------------------------------------------------------------------------
def test_graph_union_batch():
    parts = []
    for i, s in enumerate([10, 12, 9, 11]):
        n, off, col = G.rmat_host(s, 16, 100 + i, True)
        parts.append((n, off, col))
    gs = [G.Graph.from_csr(n, o, c, dir=G.InOut, symmetric=True) for n, o, c in parts]
    for g in gs:
        g.set_weights_hash(5)
    U, voff = G.Graph.union(gs)
    assert U.n == sum(p[0] for p in parts) and U.symmetric
    roots = [int(G.sample_sources(p[1], 1, 1)[0]) for p in parts]
    lv, _ = G.bfs_multiroot(U, [r + int(voff[i]) for i, r in enumerate(roots)])
    lab, _ = G.cc(U)
    pr, _ = G.pagerank(U, G.PR_ITER, 0.85, 20)
    for i, (n, off, col) in enumerate(parts):
        a, b = int(voff[i]), int(voff[i + 1])
        R = O.Restatement.from_csr(n, off, col)
        np.testing.assert_array_equal(lv[a:b], R.bfs(roots[i])[0])
        ref_lab, _ = R.cc()
        np.testing.assert_array_equal(lab[a:b] - a, ref_lab)
        ref_pr, _ = R.pagerank(1, 0.85, 20)
        assert rel_l1(pr[a:b], ref_pr) <= TOL


# ---------------------------------------------------------------------------------------------
# relabelled graphs: rows are stored sorted by internal id; per-arc data keeps the caller's order
# ---------------------------------------------------------------------------------------------
def _multigraph(n, m, seed):
    """Directed multigraph in caller CSR order with parallel arcs and self loops, unsorted rows."""
    rng = np.random.default_rng(seed)
    src = np.minimum(rng.zipf(1.6, m) - 1, n - 1).astype(np.int64)
    dst = rng.integers(0, n, m)
    dst[: m // 10] = dst[m // 10: 2 * (m // 10)]  # parallel arcs
    src[: m // 10] = src[m // 10: 2 * (m // 10)]
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order]
    off = np.zeros(n + 1, np.uint64)
    np.add.at(off, src + 1, 1)
    return n, np.cumsum(off).astype(np.uint64), dst.astype(np.uint32)


def test_relabelled_arc_order_roundtrip():
    n, off, col = _multigraph(3000, 40000, 5)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, reorder=True)
    o2, c2 = g.csr()
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(c2, col)


@pytest.mark.parametrize("when", ["weights_after_relabel", "weights_before_relabel"])
def test_relabelled_explicit_weights_match_plain(when):
    n, off, col = _multigraph(3000, 40000, 6)
    w = np.random.default_rng(7).integers(1, 1000, len(col)).astype(np.uint32)
    plain = G.Graph.from_csr(n, off, col, dir=G.InOut)
    plain.loadEdgeProperty(w)
    if when == "weights_after_relabel":
        rel = G.Graph.from_csr(n, off, col, dir=G.InOut, reorder=True)
        rel.loadEdgeProperty(w)
    else:
        rel = G.Graph.from_csr(n, off, col, dir=G.InOut)
        rel.loadEdgeProperty(w)
        rel.reorder()
    roots = np.array([0, 1, 17, 2999], np.uint32)
    d0, _ = G.sssp(plain, roots)
    d1, _ = G.sssp(rel, roots)
    np.testing.assert_array_equal(d1, d0)
    d2, _, _ = G.vc_sssp(rel, 17)
    np.testing.assert_array_equal(d2, d0.reshape(len(roots), n)[2])


@pytest.mark.parametrize("schedule", ["1,16,64,0", "2,32,256,1024", "8,128,4096,4096", "4,4096,65536,0", "2,32,64,512",
                                      "16,256,512,0", "16,65536,131072,0"])
@pytest.mark.parametrize("directed", [False, True], ids=["sym", "dir"])
def test_forced_row_schedules_match_oracle(monkeypatch, schedule, directed):
    """Every row kernel (lanes, CTA, fixed chunks, source-window chunks) gives the oracle's sums;
    SSSP too, on the schedule's bins or (more than 8 arcs per lane, or a warp above 16384 arcs) on
    its own narrower ones."""
    n, off, col = G.rmat_host(14, 16, 42, not directed)
    R = O.Restatement.from_csr(n, off, col)
    monkeypatch.setenv("GRE_ROW_SCHEDULE", schedule)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=not directed, reorder=True)
    sched = tuple(int(x) for x in schedule.split(","))
    got = g.row_schedule()
    assert got[:3] == sched[:3] and got[3] in (0, sched[3])  # no window cut when no row is above cta_min
    ref, _ = R.pagerank(1, 0.85, 20)
    pr, _ = G.pagerank(g, G.PR_ITER, 0.85, 20)
    assert rel_l1(pr, ref) <= TOL
    if not directed:
        lab, _ = G.cc(g)
        np.testing.assert_array_equal(lab, R.cc()[0])
    # SSSP with every pass through the bins (CTA rows and hub chunks, under window schedules too)
    monkeypatch.setenv("GRE_SSSP_BINNED", "4294967296")
    g.set_weights_hash(6)
    roots = G.sample_sources(off, 2, 7)
    ref = R.sssp_many(roots, 6)
    for pull in ("0", "1"):
        monkeypatch.setenv("GRE_SSSP_PULL", pull)
        np.testing.assert_array_equal(G.sssp(g, roots)[0].reshape(2, n), ref)
    w = np.exp(np.random.default_rng(3).standard_normal(len(col)))
    g.set_weights_f64(w)
    r1, _, _ = G.pagerank_weighted(g, 0.85, None, tol=1e-14, max_iters=500)
    monkeypatch.setenv("GRE_ROW_SCHEDULE", "4,4096,65536,0")
    g0 = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=not directed, reorder=True)
    g0.set_weights_f64(w)
    r0, _, _ = G.pagerank_weighted(g0, 0.85, None, tol=1e-14, max_iters=500)
    assert rel_l1(r1, r0) <= 1e-12


def test_autotuned_row_schedule_keeps_results(monkeypatch):
    """The tuner picks a schedule from its candidates; results equal the default schedule's
    (bit-exact for BFS/CC, FP64 sums within a few ulps: only the association order differs)."""
    g = G.Graph.rmat(20, 16, 77, True, reorder=True)
    lane_arcs, cta_min, hub, _ = g.row_schedule()
    assert lane_arcs in (2, 4, 8, 16) and cta_min in (4096, 16384, 65536)
    assert hub == (2 * cta_min if cta_min > 32768 else 65536)
    monkeypatch.setenv("GRE_TUNE", "0")
    g0 = G.Graph.rmat(20, 16, 77, True, reorder=True)
    assert g0.row_schedule() == (4, 4096, 65536, 0)
    pr, _ = G.pagerank(g, G.PR_ITER, 0.85, 20)
    pr0, _ = G.pagerank(g0, G.PR_ITER, 0.85, 20)
    assert rel_l1(pr, pr0) <= 1e-13
    off, _ = g.csr()
    roots = G.sample_sources(off, 64, 3)
    np.testing.assert_array_equal(G.msbfs(g, roots)[0], G.msbfs(g0, roots)[0])
    np.testing.assert_array_equal(G.cc(g)[0], G.cc(g0)[0])


# ---------------------------------------------------------------------------------------------
# scale 20: size-independent properties
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def rmat20():
    g = G.Graph.rmat(20, 16, 2024, True, reorder=True)
    off, col = g.csr()
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(off.astype(np.int64)))
    return g, off, col, src


def test_s20_bfs_properties(rmat20):
    g, off, col, src = rmat20
    roots = G.sample_sources(off, 2, 4)
    lv, _ = G.bfs(g, roots)
    lv = lv.reshape(len(roots), g.n)
    lv2, _ = G.msbfs(g, roots)
    np.testing.assert_array_equal(lv2.reshape(len(roots), g.n), lv)
    for i, r in enumerate(roots):
        L = lv[i].astype(np.int64)
        assert L[r] == 0
        a, b = L[src], L[col]
        reached = a >= 0
        assert np.all((b >= 0)[reached])  # a reached vertex's neighbours are reached
        assert np.all(np.abs(a[reached] - b[reached]) <= 1)
        # every reached vertex other than the root has a neighbour one level up
        has_parent = np.zeros(g.n, dtype=bool)
        has_parent[col[(b == a + 1) & reached]] = True
        assert np.all(has_parent[(L > 0)])


def test_s20_sssp_properties(rmat20):
    """A complete certificate of the distances at scale 20: no arc can shorten a distance (every
    arc checked), every reached vertex other than the root has a tight arc, and the reached set
    is the BFS's.  The weights are recomputed on the host by the oracle's restatement."""
    g, off, col, src = rmat20
    g.set_weights_hash(31)
    r = int(G.sample_sources(off, 1, 8)[0])
    d, _ = G.sssp(g, [r])
    wt = O.sssp_weights_csr(31, off, col).astype(np.int64)
    du, dv = d[src].astype(np.int64), d[col].astype(np.int64)
    inf = 0xFFFFFFFF
    assert d[r] == 0
    fin = du != inf
    assert np.all(dv[fin] <= du[fin] + wt[fin])
    tight = np.zeros(g.n, dtype=bool)
    tight[col[fin & (dv == du + wt)]] = True
    reached = d != inf
    reached[r] = False
    assert np.all(tight[reached])
    dl, _ = G.bfs(g, [r])
    assert np.all((d == inf) == (dl < 0))


def cc_certificate(g, lab, src, col):
    """Labels are the minimum-id labelling of the components: (1) constant along every arc,
    (2) no larger than the vertex's own id, (3) the label's vertex is labelled with itself, and (4)
    a BFS from all self-labelled vertices reaches every vertex.  By (1) a vertex reached from r
    carries r's label r, so (4) puts every vertex's label inside its own component, and (2) then
    makes it the component's smallest id.  (Without (4), two components could share one label.)"""
    ids = np.arange(g.n)
    assert np.all(lab[src] == lab[col])
    assert np.all(lab <= ids)
    assert np.all(lab[lab] == lab)
    roots = np.flatnonzero(lab == ids).astype(np.uint32)
    lv, _ = G.bfs_multiroot(g, roots)
    assert np.all(lv >= 0)


def test_s20_cc_properties(rmat20):
    g, off, col, src = rmat20
    lab, _ = G.cc(g)
    cc_certificate(g, lab, src, col)
    lab2, _ = G.vc_cc(g)
    np.testing.assert_array_equal(lab, lab2)


@pytest.mark.parametrize("pull_arcs", ["0", "16", "4294967296"], ids=["by-members", "by-arcs", "heavy-always"])
@pytest.mark.parametrize("pull", ["0", "1"], ids=["push", "pull"])
@pytest.mark.parametrize("binned", ["0", "4294967296", "64"], ids=["tiles", "bins", "default"])
def test_sssp_relaxation_forms_agree(monkeypatch, binned, pull, pull_arcs):
    """Arc tiles only, degree bins only (every pass, pushed along the frontier's arcs or pulled
    by the vertices that can improve), and the default mix give the oracle's distances; heavy
    passes pull by the bucket's member count only, also by its heavy arcs, or (almost) always."""
    monkeypatch.setenv("GRE_SSSP_BINNED", binned)
    monkeypatch.setenv("GRE_SSSP_PULL", pull)
    monkeypatch.setenv("GRE_SSSP_PULL_ARCS", pull_arcs)
    for sym in (True, False):
        n, off, col = G.rmat_host(12, 16, 9, sym)
        g = G.Graph.from_csr(n, off, col, dir=G.InOut if sym else G.Out, symmetric=sym, reorder=True)
        g.set_weights_hash(3)
        R = O.Restatement.from_csr(n, off, col)
        roots = G.sample_sources(off, 3, 1)
        ref = R.sssp_many(roots, 3)
        np.testing.assert_array_equal(G.sssp(g, roots)[0].reshape(len(roots), n), ref)


@pytest.mark.parametrize("name", SYM)
@REORDER
def test_plugin_output_statistics(golden, name, reorder):
    """The engine calls each plugin's output_statistics once after the last superstep
    (Engine.hpp:404): PageRank reports the sum of its ranks, CountIn the number of in-edges, CC the
    number of components, as the reference plugins print them."""
    case = golden[name]
    g = graph_of(case, reorder)
    pr, st = G.vc_pagerank(g, G.PR_REFERENCE, 10)
    assert abs(st.plugin_value - float(np.sum(case["pr_gre10"]))) <= 1e-12 * float(np.sum(case["pr_gre10"]))
    cn, st = G.vc_count_in(g, G.In, 1)
    assert st.plugin_count == int(case["countin"].astype(np.int64).sum())
    lab, st = G.vc_cc(g)
    assert st.plugin_count == int(np.sum(case["cc_label"] == np.arange(int(case["n"]))))
    _, st = G.cc(g)  # the fast paths run no plugin
    assert st.plugin_count == 0 and st.plugin_value == 0.0


@pytest.mark.parametrize("pull", ["0", "1"], ids=["push", "pull"])
def test_sssp_pull_needs_symmetric_weights(monkeypatch, pull):
    """The pull form reads w(v->u) for the arc u->v: it runs only where the weights are a function
    of the undirected edge (hash weights), and explicit per-arc weights that differ between the two
    directions still give the oracle's distances (push form) with every pass through the bins."""
    monkeypatch.setenv("GRE_SSSP_PULL", pull)
    monkeypatch.setenv("GRE_SSSP_BINNED", "4294967296")  # every pass through the bins
    n, off, col = G.rmat_host(13, 16, 5, True)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 4, 2)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True, reorder=True)
    w = np.random.default_rng(9).integers(1, 256, len(col)).astype(np.uint32)  # not symmetric
    g.loadEdgeProperty(w)
    np.testing.assert_array_equal(G.sssp(g, roots)[0].reshape(len(roots), n), R.sssp_many(roots, 0, w))
    g.set_weights_hash(4)
    np.testing.assert_array_equal(G.sssp(g, roots)[0].reshape(len(roots), n), R.sssp_many(roots, 4))
    for d in ("0", "1", "300"):  # Bellman-Ford frontier, unit buckets, one bucket holding everything
        monkeypatch.setenv("GRE_SSSP_DELTA", d)
        np.testing.assert_array_equal(G.sssp(g, roots)[0].reshape(len(roots), n), R.sssp_many(roots, 4))
