// Batches of graphs of uneven size in one launch sequence (gre_graph_batch_run).
//
// The reference runs one engine per graph (a driver loop around usr/test_*.cpp).  Here the k
// members become one block-diagonal union (gre_graph_union: ids of member i shifted by its vertex
// offset, no arc between members) and the algorithm runs once over it: every superstep covers all
// members, so small graphs share launches instead of each paying a full superstep's fixed cost.
// Results are cut back per member (member ids, member order).
#include <vector>

#include "gre_internal.cuh"

namespace gre {
namespace {

// labels of the union -> member ids (subtract the member's vertex offset)
__global__ void k_shift_down(uint64_t n, uint32_t* __restrict__ x, uint32_t by) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) x[i] -= by;
}

struct DeviceBuffer {
  void* p = nullptr;
  ~DeviceBuffer() { cudaFree(p); }
};

}  // namespace
}  // namespace gre

using namespace gre;

extern "C" {

int gre_graph_batch_run(const gre_graph* gs, uint32_t k, int algo, const void* params, void** outs, gre_stats* st) {
  if (!gs || !outs || k == 0) return GRE_NULL;
  for (uint32_t i = 0; i < k; ++i)
    if (!gs[i] || (!outs[i] && gs[i]->n)) return GRE_NULL;
  if (algo != GRE_BATCH_BFS && algo != GRE_BATCH_CC && algo != GRE_BATCH_PAGERANK) {
    set_error("gre_graph_batch_run: unknown algorithm %d", algo);
    return GRE_INVALID_ARG;
  }
  if ((algo == GRE_BATCH_BFS || algo == GRE_BATCH_PAGERANK) && !params) return GRE_NULL;
  std::vector<uint32_t> roots;
  if (algo == GRE_BATCH_BFS) {  // one root per member, member ids (host or device array)
    roots.resize(k);
    GRE_CUDA(cudaMemcpy(roots.data(), params, sizeof(uint32_t) * k, cudaMemcpyDefault));
    for (uint32_t i = 0; i < k; ++i)
      if (roots[i] >= gs[i]->n) {
        set_error("gre_graph_batch_run: root %u of member %u out of range (n = %llu)", roots[i], i,
                  (unsigned long long)gs[i]->n);
        return GRE_INVALID_ARG;
      }
  }
  std::vector<uint64_t> voff(k + 1);
  gre_graph u = nullptr;
  GRE_CHECK(gre_graph_union(gs, k, gs[0]->device, &u, voff.data()));
  GraphGuard guard{u};
  GRE_CHECK(use_graph(u));
  const uint64_t n = u->n;
  const size_t elem = algo == GRE_BATCH_PAGERANK ? sizeof(double) : sizeof(uint32_t);
  DeviceBuffer out;
  GRE_CUDA(cudaMalloc(&out.p, elem * (n ? n : 1)));
  if (algo == GRE_BATCH_BFS) {
    for (uint32_t i = 0; i < k; ++i) roots[i] += (uint32_t)voff[i];
    GRE_CHECK(gre_bfs_multiroot(u, roots.data(), k, (int32_t*)out.p, st));
  } else if (algo == GRE_BATCH_CC) {
    GRE_CHECK(gre_cc(u, (uint32_t*)out.p, st));
    for (uint32_t i = 0; i < k; ++i)
      if (voff[i + 1] > voff[i] && voff[i])
        k_shift_down<<<grid_for(voff[i + 1] - voff[i], 256), 256, 0, u->stream>>>(voff[i + 1] - voff[i],
                                                                                  (uint32_t*)out.p + voff[i], (uint32_t)voff[i]);
    GRE_LAUNCH_CHECK();
  } else {
    const gre_batch_pagerank_params* pp = (const gre_batch_pagerank_params*)params;
    GRE_CHECK(gre_pagerank(u, pp->variant, pp->d, pp->iters, (double*)out.p, st));
  }
  GRE_CUDA(cudaStreamSynchronize(u->stream));
  for (uint32_t i = 0; i < k; ++i) {
    const uint64_t ni = voff[i + 1] - voff[i];
    if (ni) GRE_CUDA(cudaMemcpy(outs[i], (const char*)out.p + elem * voff[i], elem * ni, cudaMemcpyDefault));
  }
  return GRE_SUCCESS;
}

}  // extern "C"
