"""The stated benchmark configs, run as stated, against the oracle and the reference itself.

* PageRank-20 on directed RMAT-16 (EF16, written as 4 edge-list files + .meta): both plugins
  against the reference engine's own run (oracle/_ref, compiled from its headers) on the same
  files, within 1e-9 relative L1.
* BFS, SSSP (uint32 weights in [1, 255]) and CC on symmetric RMAT-22 from 16 seeded
  non-isolated sources: levels, distances and min-labels bit-exact against the oracle's
  restatement (pinned to the reference by the golden fixtures), and one source of each
  against the reference engine itself at scale 18.
* Batched at scale 20: 256-source BC batched == looped (bit for bit) and within 1e-9 of the
  oracle on a sample of sources; 64-source BFS against the oracle; 128 personalised PageRank
  vectors batched against looped and against the oracle for a sample; 32 RMAT graphs of
  scales 12-18 in one union against per-graph oracle runs.
"""
import os
import tempfile

import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O
from conftest import rel_l1

pytestmark = pytest.mark.gpu
TOL = 1e-9
WSEED = 20240601

needs_reference = pytest.mark.skipif(not O.reference_available(), reason="reference binaries not built (oracle/_ref)")


# ---------------------------------------------------------------------------------------------
# PageRank-20, directed RMAT-16, text files: against the reference engine's own run
# ---------------------------------------------------------------------------------------------
@needs_reference
def test_pagerank_s16_directed_vs_reference_engine():
    n, off, col = O.rmat(16, 16, 1, False)
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, "pr16")
        O.write_edgelists(prefix, n, off, col, 4)
        g = G.Graph.ingress(prefix, G.Out, reorder=True)
        for variant, name in ((G.PR_REFERENCE, "gre"), (G.PR_ITER, "iter")):
            ref, run = O.run_reference("pagerank", prefix, name, 20, 1)
            pr, st = G.pagerank(g, variant, 0.85, 20)
            assert rel_l1(pr, ref[:n]) <= TOL, name
            assert st.traversed_edges == g.m * 20
            pv, sv = G.vc_pagerank(g, variant, 20)  # the device engine: same active counts too
            assert rel_l1(pv, ref[:n]) <= TOL and sv.active == run.active[0]


# ---------------------------------------------------------------------------------------------
# BFS / SSSP / CC, symmetric RMAT-22, 16 sources
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def s22():
    n, off, col = G.rmat_host(22, 16, 22, True)
    g = G.Graph.rmat(22, 16, 22, True, reorder=True)  # the same graph, generated on the device
    g.set_weights_hash(WSEED)
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 16, 22)
    return n, off, col, g, R, roots


def test_s22_bfs_16_sources_bit_exact(s22):
    n, off, col, g, R, roots = s22
    ref = R.bfs_many(roots)
    lv, st = G.bfs(g, roots)
    np.testing.assert_array_equal(lv.reshape(16, n), ref)
    lv, _ = G.msbfs(g, roots)
    np.testing.assert_array_equal(lv.reshape(16, n), ref)


def test_s22_sssp_16_sources_bit_exact(s22):
    n, off, col, g, R, roots = s22
    ref = R.sssp_many(roots, WSEED)
    d, _ = G.sssp(g, roots)
    np.testing.assert_array_equal(d.reshape(16, n), ref)


def test_s22_cc_bit_exact(s22):
    n, off, col, g, R, roots = s22
    ref, _ = R.cc()
    lab, _ = G.cc(g)
    np.testing.assert_array_equal(lab, ref)


@needs_reference
def test_s18_one_source_each_vs_reference_engine():
    """BFS levels, SSSP distances and CC labels against the reference engine itself (text files
    in, its own ingress; -O0 as its Makefile builds it, so scale 18 keeps this to seconds)."""
    n, off, col = O.rmat(18, 16, 18, True)
    roots = O.sample_sources(off, 1, 18)
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, "s18")
        O.write_edgelists(prefix, n, off, col, 4)
        O.write_roots(prefix, roots)
        g = G.Graph.ingress(prefix, G.InOut, symmetric=True, reorder=True)
        g.set_weights_hash(WSEED)
        ref_lv, _ = O.run_reference("bfs", prefix, 1)
        ref_d, _ = O.run_reference("sssp", prefix, WSEED, 1)
        ref_cc, _ = O.run_reference("cc", prefix)
    lv, _ = G.bfs(g, roots)
    np.testing.assert_array_equal(lv, ref_lv[:n])
    d, _ = G.sssp(g, roots)
    np.testing.assert_array_equal(d, ref_d[:n])
    lab, _ = G.cc(g)
    np.testing.assert_array_equal(lab.astype(np.uint64), ref_cc[:n])


# ---------------------------------------------------------------------------------------------
# batched forms at scale 20
# ---------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def s20():
    n, off, col = G.rmat_host(20, 16, 77, True)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True, reorder=True)
    R = O.Restatement.from_csr(n, off, col)
    return n, off, col, g, R


def test_s20_bc_256_batched_equals_looped_and_oracle(s20):
    n, off, col, g, R = s20
    srcs = G.sample_sources(off, 256, 11)
    b_loop, _ = G.bc(g, srcs, batched=False)
    b_bat, _ = G.bc(g, srcs, batched=True)
    np.testing.assert_array_equal(b_bat, b_loop)
    few = srcs[::32]  # 8 of the sources through the oracle
    ref, _ = R.bc(few)
    got, _ = G.bc(g, few, batched=True)
    assert rel_l1(got, ref) <= TOL


def test_s20_bfs_64_sources(s20):
    n, off, col, g, R = s20
    srcs = G.sample_sources(off, 64, 12)
    ref = R.bfs_many(srcs)
    lv, _ = G.msbfs(g, srcs)
    np.testing.assert_array_equal(lv.reshape(64, n), ref)


def test_s20_ppr_128_vectors(s20):
    n, off, col, g, R = s20
    seeds = G.sample_sources(off, 128, 13)
    a, _ = G.ppr(g, seeds, 0.85, 20, batched=True)
    b, _ = G.ppr(g, seeds, 0.85, 20, batched=False)
    assert rel_l1(a, b) <= TOL
    few = seeds[::16]
    ref = R.ppr(few, 0.85, 20)
    assert rel_l1(a.reshape(128, n)[::16], ref) <= TOL


def test_graph_batch_32_uneven_scales():
    rng = np.random.default_rng(77)
    scales = rng.integers(12, 19, size=32)
    parts = [G.rmat_host(int(s), 16, 77 + i, True) for i, s in enumerate(scales)]
    gs = [G.Graph.from_csr(n, o, c, dir=G.InOut, symmetric=True) for n, o, c in parts]
    roots = [int(G.sample_sources(o, 1, 3)[0]) for _, o, _ in parts]
    lv, _ = G.graph_batch_run(gs, G.BATCH_BFS, roots=roots)
    lab, _ = G.graph_batch_run(gs, G.BATCH_CC)
    for i, (n, o, c) in enumerate(parts):
        R = O.Restatement.from_csr(n, o, c)
        np.testing.assert_array_equal(lv[i], R.bfs(roots[i])[0])
        np.testing.assert_array_equal(lab[i], R.cc()[0])
