"""The 64-source BFS as one persistent launch (persist.cu).

* The cooperative level loop gives the levels of the host-driven loop bit for bit (and the
  oracle's), with the same per-level counts of new (source, vertex) pairs.
* A grid-barrier wait that runs out ends the launch with GRE_TIMEOUT and leaves the context and
  the graph usable: the budget is set to 0 (every wait fails at once; nothing faults or hangs),
  then the same call with the default budget gives the right levels.
"""
import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [1, 64, 70])
def test_persistent_levels_equal_host_loop_and_oracle(monkeypatch, k):
    n, off, col = G.rmat_host(16, 16, 31, True)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True, reorder=True)
    srcs = G.sample_sources(off, k, 4)
    monkeypatch.setenv("GRE_PERSIST", "0")
    host, st_host = G.msbfs(g, srcs)
    monkeypatch.setenv("GRE_PERSIST", "1")
    pers, st_pers = G.msbfs(g, srcs)
    np.testing.assert_array_equal(pers, host)
    assert st_pers.active == st_host.active and st_pers.supersteps == st_host.supersteps
    assert st_pers.arcs_traversed == st_host.arcs_traversed
    R = O.Restatement.from_csr(n, off, col)
    np.testing.assert_array_equal(pers.reshape(len(srcs), n), R.bfs_many(srcs))


def test_persistent_wait_budget_runs_out_cleanly(monkeypatch):
    n, off, col = G.rmat_host(14, 16, 32, True)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True)
    srcs = G.sample_sources(off, 64, 5)
    monkeypatch.setenv("GRE_PERSIST", "1")
    monkeypatch.setenv("GRE_GRID_WAIT_MS", "0")
    with pytest.raises(G.GreError) as e:
        G.msbfs(g, srcs)
    assert e.value.status == G.GRE_TIMEOUT
    assert "grid barrier" in str(e.value)
    monkeypatch.delenv("GRE_GRID_WAIT_MS")
    lv, _ = G.msbfs(g, srcs)  # the same graph, the same context: a normal run
    np.testing.assert_array_equal(lv.reshape(64, n), O.Restatement.from_csr(n, off, col).bfs_many(srcs))


def test_batched_graphs_bfs_persistent_equals_host_loop(monkeypatch):
    """A batch of uneven graphs (one block-diagonal union, one root each) through the persistent
    level loop (on request: GRE_PERSIST=1), the roots sharing one source bit: levels, per-level
    counts, supersteps and reached edges equal the host-driven direction-optimising BFS's, and
    each member's levels the oracle's."""
    parts = [G.rmat_host(s, 8, 60 + i, True) for i, s in enumerate([12, 9, 14, 11, 13])]
    gs = [G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True) for n, off, col in parts]
    U, voff = G.Graph.union(gs)
    roots = [int(G.sample_sources(off, 1, i)[0]) + int(voff[i]) for i, (n, off, col) in enumerate(parts)]
    monkeypatch.setenv("GRE_PERSIST", "0")
    host, st_host = G.bfs_multiroot(U, roots)
    monkeypatch.setenv("GRE_PERSIST", "1")
    pers, st_pers = G.bfs_multiroot(U, roots)
    np.testing.assert_array_equal(pers, host)
    assert st_pers.active == st_host.active and st_pers.supersteps == st_host.supersteps
    assert st_pers.traversed_edges == st_host.traversed_edges
    for i, (n, off, col) in enumerate(parts):
        a, b = int(voff[i]), int(voff[i + 1])
        ref = O.Restatement.from_csr(n, off, col).bfs(roots[i] - a)[0]
        np.testing.assert_array_equal(pers[a:b], ref)
