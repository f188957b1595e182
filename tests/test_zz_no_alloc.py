"""gre_bfs_noalloc: the BFS entry point that allocates no device memory.

It exists for callers that cannot let a library allocate: a process whose device memory is
reserved up front and capped by its own pool allocator (a cudaMalloc outside the pool fails or
breaks the budget), or a latency-critical loop that cannot take the implicit device
synchronisation of cudaMalloc / cudaFree.  Its scratch is a fixed array inside the library.

Checked through the C ABI: the levels equal those of gre_bfs (bit-exact, as every integer
result here) on two calls in a row that share the scratch, on a plain and a relabelled graph;
the calls change no free device memory; graphs beyond the scratch's 1,048,576 vertices and
output buffers that are not device memory of the graph's device (pageable or pinned host memory)
are rejected.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import graphine_b200.gre as G

pytestmark = pytest.mark.gpu


def noalloc_bfs(g, src, out):
    st = G._Stats()
    rc = G.lib().gre_bfs_noalloc(g._h, int(src), out.data_ptr(), ctypes.byref(st))
    assert rc == G.GRE_SUCCESS, G.last_error()
    return st


@pytest.mark.parametrize("reorder", [False, True], ids=["plain", "relabelled"])
def test_noalloc_bfs_equals_gre_bfs_on_consecutive_calls(reorder):
    import torch

    n, off, col = G.rmat_host(16, 16, 12, True)
    g = G.Graph.from_csr(n, off, col, dir=G.InOut, symmetric=True, reorder=reorder)
    srcs = G.sample_sources(off, 2, 3)
    outs = [torch.empty(n, dtype=torch.int32, device="cuda") for _ in srcs]
    noalloc_bfs(g, srcs[0], outs[0])  # first call on the device: looks up the scratch address
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for s, out in zip(srcs, outs):  # two calls in a row, the second reusing the first's scratch
        st = noalloc_bfs(g, s, out)
        assert st.supersteps > 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    for s, out in zip(srcs, outs):
        ref, _ = G.bfs(g, [s])
        np.testing.assert_array_equal(out.cpu().numpy(), ref)


def test_noalloc_rejects_oversize_graph_and_host_output():
    import torch

    big = G.Graph.rmat(21, 2, 1, True)  # 2,097,152 vertices
    out = torch.empty(big.n, dtype=torch.int32, device="cuda")
    assert G.lib().gre_bfs_noalloc(big._h, 0, out.data_ptr(), None) == G.GRE_INVALID_ARG
    assert "1048576" in G.last_error()
    small = G.Graph.rmat(10, 8, 1, True)
    host = np.empty(small.n, dtype=np.int32)
    assert G.lib().gre_bfs_noalloc(small._h, 0, host.ctypes.data, None) == G.GRE_INVALID_ARG
    pinned = torch.empty(small.n, dtype=torch.int32, pin_memory=True)  # host memory the GPU can map
    assert G.lib().gre_bfs_noalloc(small._h, 0, pinned.data_ptr(), None) == G.GRE_INVALID_ARG
    assert "graph's device" in G.last_error()
