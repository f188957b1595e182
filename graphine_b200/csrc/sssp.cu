// SSSP fast path: frontier relaxation with uint32 weights.
//
// Same fixed point as the reference SSSP plugin (Kernels/SSSP.hpp:55-89: scatter last[u]+w,
// combine = min, every improved vertex re-activated): shortest-path distances are unique, so
// the result is bit-exact whatever the relaxation order.  Differences from the reference's
// superstep, chosen for the GPU:
//   * the frontier is a queue of improved vertices, expanded edge-balanced (one thread per
//     frontier arc, owner found by binary search in the scan of frontier degrees), so hubs do
//     not serialise a warp;
//   * the distance of the frontier vertex is read when its arc is relaxed (not a copy taken
//     at the start of the superstep), which can only lower the values sent and converges in
//     at most as many supersteps;
//   * a bitmap de-duplicates the next frontier (one queue slot per improved vertex).
//
// Byte model per superstep: 16 F (queue + offsets) + 12 A (column + weight + dist probe)
// + 8 N (queue append + bitmap), F frontier, A arcs relaxed, N improved vertices.
#include <cub/cub.cuh>

#include <algorithm>

#include "gre_internal.cuh"

namespace gre {

template <class T>
static int ws_array(gre_graph g, int slot, uint64_t count, T** p) {
  void* v = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &v));
  *p = (T*)v;
  return GRE_SUCCESS;
}

__global__ void k_sssp_seed(uint32_t src, uint32_t* __restrict__ dist, uint32_t* __restrict__ queue) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    dist[src] = 0;
    queue[0] = src;
  }
}

__global__ void k_sssp_degrees(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ off,
                               uint64_t* __restrict__ deg) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = queue[i];
    deg[i] = off[u + 1] - off[u];
  }
}

__global__ void __launch_bounds__(256) k_sssp_relax(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ prefix,
                                                    uint64_t total, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                    const uint32_t* __restrict__ w, uint32_t* __restrict__ dist,
                                                    uint32_t* __restrict__ inq, uint32_t* __restrict__ next_queue,
                                                    uint32_t* __restrict__ next_count) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < total; base += stride) {
    const uint64_t t = base + (threadIdx.x & 31u);
    bool push = false;
    uint32_t v = 0;
    if (t < total) {
      uint64_t lo = 0, hi = nq;
      while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= t) lo = mid;
        else hi = mid;
      }
      const uint32_t u = queue[lo];
      const uint64_t a = off[u] + (t - prefix[lo]);
      v = __ldg(col + a);
      const uint32_t nd = *(volatile uint32_t*)(dist + u) + __ldg(w + a);
      if (nd < *(volatile uint32_t*)(dist + v)) {
        const uint32_t old = atomicMin(dist + v, nd);
        if (nd < old) {
          const uint32_t bit = 1u << (v & 31u);
          const uint32_t prev = atomicOr(inq + (v >> 5), bit);
          push = !(prev & bit);
        }
      }
    }
    const uint32_t pos = warp_append(next_count, push);
    if (push) next_queue[pos] = v;
  }
}

__global__ void k_sssp_clear_bits(const uint32_t* __restrict__ queue, uint64_t nq, uint32_t* __restrict__ inq) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = queue[i];
    atomicAnd(inq + (v >> 5), ~(1u << (v & 31u)));
  }
}

static int sssp_one(gre_graph g, uint32_t src, uint32_t* dist, gre_stats* st, bool record) {
  const uint64_t n = g->n;
  const uint64_t nwords = (n + 31) >> 5;
  uint32_t *qa, *qb, *inq, *cnt;
  uint64_t *deg, *prefix;
  GRE_CHECK(ws_array(g, WS_A, n, &qa));
  GRE_CHECK(ws_array(g, WS_B, n, &qb));
  GRE_CHECK(ws_array(g, WS_C, nwords, &inq));
  GRE_CHECK(ws_array(g, WS_F, n + 1, &deg));
  GRE_CHECK(ws_array(g, WS_G, n + 1, &prefix));
  GRE_CHECK(ws_array(g, WS_COUNTERS, 4, &cnt));
  size_t cubbytes = 0;
  void* cubtmp = nullptr;
  cub::DeviceScan::ExclusiveSum(nullptr, cubbytes, deg, prefix, n + 1, g->stream);
  GRE_CHECK(g->ws.get(WS_CUB, cubbytes, &cubtmp));
  GRE_CUDA(cudaMemsetAsync(dist, 0xff, sizeof(uint32_t) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(inq, 0, sizeof(uint32_t) * nwords, g->stream));
  k_sssp_seed<<<1, 32, 0, g->stream>>>(src, dist, qa);
  uint64_t nq = 1, relaxed = 0, bytes = 0;
  uint32_t* q = qa;
  uint32_t* nqueue = qb;
  uint32_t steps = 0;
  const int sms = num_sms();
  while (nq > 0) {
    k_sssp_degrees<<<grid_for(nq, 256), 256, 0, g->stream>>>(q, nq, g->off, deg);
    GRE_CUDA(cub::DeviceScan::ExclusiveSum(cubtmp, cubbytes, deg, prefix, nq + 1, g->stream));
    GRE_CUDA(cudaMemsetAsync(cnt, 0, 4, g->stream));
    uint64_t total = 0;
    GRE_CUDA(cudaMemcpyAsync(&total, prefix + nq, sizeof total, cudaMemcpyDeviceToHost, g->stream));
    GRE_CUDA(cudaStreamSynchronize(g->stream));
    // vertices leave the queue: they may be re-queued by this superstep's relaxations
    k_sssp_clear_bits<<<grid_for(nq, 256), 256, 0, g->stream>>>(q, nq, inq);
    if (total) {
      const int grid = (int)std::min<uint64_t>((total + 255) / 256, (uint64_t)sms * 16);
      k_sssp_relax<<<grid, 256, 0, g->stream>>>(q, nq, prefix, total, g->off, g->col, g->w32, dist, inq, nqueue, cnt);
    }
    GRE_LAUNCH_CHECK();
    uint32_t h = 0;
    GRE_CUDA(cudaMemcpyAsync(&h, cnt, 4, cudaMemcpyDeviceToHost, g->stream));
    GRE_CUDA(cudaStreamSynchronize(g->stream));
    relaxed += total;
    bytes += 16 * nq + 12 * total + 8 * (uint64_t)h;
    nq = h;
    std::swap(q, nqueue);
    ++steps;
    if (record) stats_record(st, nq);
  }
  if (st) {
    st->supersteps += steps ? steps - 1 : 0;
    st->arcs_traversed += relaxed;
    st->algo_bytes += bytes;
  }
  return GRE_SUCCESS;
}

__global__ void k_dist_to_level(uint64_t n, const uint32_t* __restrict__ dist, int32_t* __restrict__ lv) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    lv[v] = dist[v] == 0xffffffffu ? -1 : 0;
}

}  // namespace gre

using namespace gre;

extern "C" {

int gre_sssp(gre_graph g, const uint32_t* srcs, uint32_t nsrc, uint32_t* dist, gre_stats* st) {
  if (!g || !dist || (nsrc && !srcs)) return GRE_NULL;
  if (!g->w32) {
    set_error("gre_sssp: the graph has no uint32 weights (gre_graph_set_weights_*)");
    return GRE_INVALID_ARG;
  }
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  std::vector<uint32_t> hs(nsrc);
  if (nsrc) GRE_CUDA(cudaMemcpy(hs.data(), srcs, sizeof(uint32_t) * nsrc, cudaMemcpyDefault));
  GRE_CHECK(map_ids(g, &hs, "gre_sssp"));
  uint32_t *dfinal, *dd;
  int32_t* lv;
  GRE_CHECK(prepare_output(g, dist, (uint64_t)nsrc * n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, nsrc, 4, (void**)&dd));
  GRE_CHECK(ws_array(g, WS_H, n, &lv));
  RunTimer timer(g);
  uint64_t edges = 0;
  for (uint32_t i = 0; i < nsrc; ++i) {
    GRE_CHECK(sssp_one(g, hs[i], dd + (uint64_t)i * n, st, nsrc == 1));
    k_dist_to_level<<<grid_for(n, 256), 256, 0, g->stream>>>(n, dd + (uint64_t)i * n, lv);
    uint64_t e = 0;
    GRE_CHECK(count_reached_edges(g, lv, &e));
    edges += e;
  }
  GRE_CHECK(perm_out_end(g, dd, dfinal, nsrc, 4));
  GRE_CHECK(finish_output(g, dist, dfinal, (uint64_t)nsrc * n));
  GRE_CHECK(timer.stop(st));
  if (st) st->traversed_edges = edges;
  return GRE_SUCCESS;
}

}  // extern "C"
