// Connected components fast path: lock-free union-find with min-id hooking.
//
// The reference ConnectedComponents plugin (Kernels/CC.hpp:33-67, run<InOut>) propagates the
// minimum global vid across every arc until no label changes; the fixed point labels each
// vertex with the minimum vid of its (weakly) connected component.  Union-find reaches the
// same labels directly: every arc {u, v} unites the two trees, and a root is only ever linked
// under a smaller root (atomicCAS on the larger root's parent), so the root of each tree is
// the minimum vid it contains.  A final pass writes find(v) for every v.  (Jayanti & Tarjan
// style concurrent union-find as used by ECL-CC, Jaiganesh & Burtscher 2018.)
//
// Arcs are visited through the degree bins of the CSR (rows.cuh): groups of 1..32 lanes per
// row, a CTA per long row, CTA chunks for hubs, so the column reads stay coalesced.  On a
// symmetric graph each undirected edge is stored twice and only the copy with v < u is used.
//
// Byte model: 8(n+1) offsets + 4m columns + 8m parent probes (two finds per arc, mostly L2)
// + 8n init/final labels.
#include "gre_internal.cuh"
#include "rows.cuh"

namespace gre {

__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x) {
  uint32_t p = parent[x];
  while (p != x) {
    const uint32_t gp = parent[p];
    if (gp != p) parent[x] = gp;  // path halving (benign race: gp is an ancestor)
    x = p;
    p = gp;
  }
  return x;
}

// key(x): the caller's vid of internal vertex x (relabelled graphs) - roots are linked by it
__device__ __forceinline__ uint32_t uf_key(const uint32_t* __restrict__ vid, uint32_t x) { return vid ? __ldg(vid + x) : x; }

__device__ __forceinline__ void uf_union(uint32_t* parent, const uint32_t* __restrict__ vid, uint32_t a, uint32_t b) {
  while (true) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return;
    const bool a_hi = uf_key(vid, a) > uf_key(vid, b);
    const uint32_t hi = a_hi ? a : b;
    const uint32_t lo = a_hi ? b : a;
    if (atomicCAS(parent + hi, hi, lo) == hi) return;
    // hi gained a parent meanwhile: retry from the new roots
    a = hi;
    b = lo;
  }
}

struct HookArcs {
  const uint32_t* __restrict__ col;
  uint32_t* parent;
  const uint32_t* __restrict__ vid;  // internal -> caller id, null when not relabelled
  bool half;                          // symmetric: use only arcs with col < row
  __device__ __forceinline__ double operator()(uint32_t u, uint64_t a) const {
    const uint32_t v = __ldg(col + a);
    if (!half || v < u) uf_union(parent, vid, u, v);
    return 0.0;
  }
};
struct NoFinish {
  __device__ __forceinline__ void operator()(uint32_t, double) const {}
};

__global__ void k_uf_init(uint64_t n, uint32_t* __restrict__ parent) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    parent[v] = (uint32_t)v;
}

// label (in caller ids) of every internal vertex: the key of its root
__global__ void k_uf_flatten(uint64_t n, uint32_t* parent, const uint32_t* __restrict__ vid, uint32_t* __restrict__ label) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    label[v] = uf_key(vid, uf_find(parent, (uint32_t)v));
}

__global__ void k_count_roots(uint64_t n, const uint32_t* __restrict__ label, unsigned long long* __restrict__ c) {
  unsigned long long s = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    s += label[v] == v;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31u) == 0 && s) atomicAdd(c, s);
}

}  // namespace gre

using namespace gre;

extern "C" {

int gre_cc(gre_graph g, uint32_t* label, gre_stats* st) {
  if (!g || !label) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  GRE_CHECK(ensure_bins(g, false));
  uint32_t *dfinal, *dl, *parent;
  double* partial;
  void* p;
  GRE_CHECK(prepare_output(g, label, n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, 1, 4, (void**)&dl));
  GRE_CHECK(g->ws.get(WS_A, sizeof(uint32_t) * n, &p));
  parent = (uint32_t*)p;
  GRE_CHECK(g->ws.get(WS_B, sizeof(double) * (g->bins_out.n_hub_chunks + 1), &p));
  partial = (double*)p;
  RunTimer timer(g);
  k_uf_init<<<grid_for(n, 256), 256, 0, g->stream>>>(n, parent);
  GRE_CHECK(rows::reduce_rows(g->bins_out, g->off, HookArcs{g->col, parent, g->perm, g->symmetric()}, NoFinish{}, partial,
                              g->stream));
  k_uf_flatten<<<grid_for(n, 256), 256, 0, g->stream>>>(n, parent, g->perm, dl);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(perm_out_end(g, dl, dfinal, 1, 4));
  GRE_CHECK(finish_output(g, label, dfinal, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = 1;
    st->arcs_traversed = g->m;
    st->traversed_edges = g->symmetric() ? g->m / 2 : g->m;
    st->algo_bytes = 8 * (n + 1) + 12 * g->m + 8 * n;
  }
  return GRE_SUCCESS;
}

}  // extern "C"
