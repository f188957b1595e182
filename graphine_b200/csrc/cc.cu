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
// row, a CTA per long row, CTA chunks for hubs, so the column reads stay coalesced.  A directed
// graph's arcs are all visited (their union is the weakly connected components).
//
// On a symmetric graph the arcs are visited the Afforest way (Sutton, Ben-Nun and Bar 2018):
// the first two arcs of every row, then the rest of the rows outside the largest component
// only; on RMAT most rows belong to it (RMAT-26: 7.8 -> 3.6 ms).
//
// Byte model: 8(n+1) offsets + 12 per visited arc (column + two parent probes, mostly L2)
// + 8n init/final labels (+ n/4 for the skip bits and their reads).
#include <algorithm>
#include <vector>

#include "gre_internal.cuh"
#include "rows.cuh"
#include "uf.cuh"

namespace gre {

struct HookArcs {
  const uint32_t* __restrict__ col;
  uint32_t* parent;
  const uint32_t* __restrict__ vid;  // internal -> caller id, null when not relabelled
  bool half;                          // symmetric: use only arcs with col < row
  // Afforest's second pass: rows flagged in `skip` are left out and the first `sampled` arcs of
  // the others were already united (null: every arc)
  const uint32_t* __restrict__ skip = nullptr;
  const uint64_t* __restrict__ off = nullptr;
  uint32_t sampled = 0;
  __device__ __forceinline__ double operator()(uint32_t u, uint64_t a) const {
    if (skip) {
      if ((__ldg(skip + (u >> 5)) >> (u & 31u)) & 1u) return 0.0;
      if (a < __ldg(off + u) + sampled) return 0.0;
    }
    const uint32_t v = __ldg(col + a);
    if (!half || v < u) uf_union(parent, vid, u, v);
    return 0.0;
  }
};

// Afforest (Sutton, Ben-Nun and Bar 2018), first pass: every vertex is united with its first k
// neighbours (relabelled rows list the hubs first, which joins most of a giant component).
__global__ void k_uf_sample(uint64_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col, uint32_t k,
                            uint32_t* parent, const uint32_t* __restrict__ vid) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n; u += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a0 = off[u], a1 = off[u + 1];
    for (uint64_t a = a0; a < a1 && a < a0 + k; ++a) uf_union(parent, vid, (uint32_t)u, __ldg(col + a));
  }
}

// parent[v] = root of v, and the roots of an evenly spaced sample of vertices
__global__ void k_uf_compress(uint64_t n, uint32_t* parent, uint64_t stride, uint32_t* __restrict__ sample, uint32_t nsample) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = uf_find(parent, (uint32_t)v);
    parent[v] = r;
    if (v % stride == 0 && v / stride < nsample) sample[v / stride] = r;
  }
}

// skip bit of every vertex already in the largest component c; counts[0] += arcs sampled,
// counts[1] += arcs the second pass still visits (byte model)
__global__ void k_uf_skipbits(uint64_t n, const uint32_t* __restrict__ parent, const uint64_t* __restrict__ off, uint32_t c,
                              uint32_t k, uint32_t* __restrict__ skip, unsigned long long* __restrict__ counts) {
  const uint64_t nwords = (n + 31) >> 5;
  unsigned long long sampled = 0, rest = 0;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    for (uint32_t b = 0; b < 32 && (w << 5) + b < n; ++b) {
      const uint64_t v = (w << 5) + b;
      const uint64_t d = off[v + 1] - off[v];
      const bool in_c = parent[v] == c;
      bits |= (uint32_t)in_c << b;
      sampled += d < k ? d : k;
      if (!in_c && d > k) rest += d - k;
    }
    skip[w] = bits;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sampled += __shfl_xor_sync(0xffffffffu, sampled, o);
    rest += __shfl_xor_sync(0xffffffffu, rest, o);
  }
  if ((threadIdx.x & 31u) == 0) {
    if (sampled) atomicAdd(counts, sampled);
    if (rest) atomicAdd(counts + 1, rest);
  }
}
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

uint32_t uf_most_frequent(std::vector<uint32_t>& hs, uint32_t ns) {
  std::sort(hs.begin(), hs.begin() + ns);
  uint32_t best = hs[0], run = 0, best_run = 0;
  for (uint32_t i = 0; i < ns; ++i) {
    run = (i && hs[i] == hs[i - 1]) ? run + 1 : 1;
    if (run > best_run) {
      best_run = run;
      best = hs[i];
    }
  }
  return best;
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
  GRE_CHECK(g->ws.get(WS_B, sizeof(double) * (g->bins_out.n_partials + 1), &p));
  partial = (double*)p;
  constexpr uint32_t kSampled = 2, kSample = 1024;
  uint32_t *skip = nullptr, *sample = nullptr;
  unsigned long long* counts = nullptr;
  if (g->symmetric()) {
    GRE_CHECK(g->ws.get(WS_C, sizeof(uint32_t) * (((n + 31) >> 5) + kSample), &p));
    skip = (uint32_t*)p;
    sample = skip + ((n + 31) >> 5);
    GRE_CHECK(g->ws.get(WS_COUNTERS, 2 * sizeof(unsigned long long), &p));
    counts = (unsigned long long*)p;
  }
  RunTimer timer(g);
  k_uf_init<<<grid_for(n, 256), 256, 0, g->stream>>>(n, parent);
  if (g->symmetric()) {
    // Afforest: unite the first arcs of every row, find the largest component from a sample,
    // then unite the remaining arcs of the vertices outside it only.  Undirected edges appear
    // in both rows, so an edge between the largest component and another vertex is seen from
    // the other side.
    k_uf_sample<<<grid_for(n, 256), 256, 0, g->stream>>>(n, g->off, g->col, kSampled, parent, g->perm);
    const uint64_t stride = n > kSample ? n / kSample : 1;
    k_uf_compress<<<grid_for(n, 256), 256, 0, g->stream>>>(n, parent, stride, sample, kSample);
    std::vector<uint32_t> hs(kSample, 0);
    const uint32_t ns = (uint32_t)std::min<uint64_t>(kSample, (n + stride - 1) / stride);
    GRE_CUDA(cudaMemcpyAsync(hs.data(), sample, sizeof(uint32_t) * ns, cudaMemcpyDeviceToHost, g->stream));
    GRE_CUDA(cudaStreamSynchronize(g->stream));
    const uint32_t best = uf_most_frequent(hs, ns);
    GRE_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), g->stream));
    k_uf_skipbits<<<grid_for((n + 31) >> 5, 256), 256, 0, g->stream>>>(n, parent, g->off, best, kSampled, skip, counts);
    HookArcs rest{g->col, parent, g->perm, false, skip, g->off, kSampled};
    GRE_CHECK(rows::reduce_rows(g->bins_out, g->off, rest, NoFinish{}, partial, g->stream));
  } else {
    GRE_CHECK(rows::reduce_rows(g->bins_out, g->off, HookArcs{g->col, parent, g->perm, false}, NoFinish{}, partial,
                                g->stream));
  }
  k_uf_flatten<<<grid_for(n, 256), 256, 0, g->stream>>>(n, parent, g->perm, dl);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(perm_out_end(g, dl, dfinal, 1, 4));
  GRE_CHECK(finish_output(g, label, dfinal, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    uint64_t visited = g->m;
    if (g->symmetric()) {  // arcs the two Afforest passes visited
      unsigned long long h[2] = {0, 0};
      GRE_CUDA(cudaMemcpy(h, counts, sizeof h, cudaMemcpyDeviceToHost));
      visited = h[0] + h[1];
    }
    st->supersteps = 1;
    st->arcs_traversed = visited;
    st->traversed_edges = g->symmetric() ? g->m / 2 : g->m;
    st->algo_bytes = 8 * (n + 1) + 12 * visited + 8 * n + (g->symmetric() ? n / 4 : 0);
  }
  return GRE_SUCCESS;
}

}  // extern "C"
