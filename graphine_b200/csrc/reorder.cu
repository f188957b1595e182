// Degree-ordered relabelling support: caller ids <-> internal ids.
//
// A relabelled graph stores vertices in order of decreasing degree (ties by id), so the
// per-vertex state of the hubs - which most arcs point to - is packed into the first few
// hundred MB and stays resident in the 126 MB L2 across a superstep's random gathers.  The
// permutation is invisible to callers: source ids are mapped on the way in, every per-vertex
// and per-arc result is un-permuted on the way out, and labels that are vertex ids (CC, BFS
// pred) are produced in caller ids directly (the reference's lvid2vid, DistributedGraph.hpp:57).
#include <cub/cub.cuh>

#include "gre_internal.cuh"

namespace gre {

template <class T>
__global__ void k_unperm(uint64_t n, uint64_t rows, const uint32_t* __restrict__ iperm, const T* __restrict__ in, T* __restrict__ out) {
  const uint64_t total = rows * n;
  for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < total; idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = idx / n, v = idx - r * n;
    out[idx] = in[r * n + iperm[v]];
  }
}

template <class T>
__global__ void k_perm(uint64_t n, const uint32_t* __restrict__ perm, const T* __restrict__ in, T* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

__global__ void k_caller_degree(uint64_t n, const uint32_t* __restrict__ iperm, const uint64_t* __restrict__ off,
                                uint64_t* __restrict__ deg) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= n; v += (uint64_t)gridDim.x * blockDim.x)
    deg[v] = v < n ? off[iperm[v] + 1] - off[iperm[v]] : 0;
}

// warp per internal row i: arc i0 + k of internal row i <-> arc c0 + rank[i0 + k] of caller row
// perm[i] (rows are sorted by internal neighbour id; rank is each arc's caller position)
template <class T, bool TO_INTERNAL>
__global__ void k_arcs(uint64_t n, const uint32_t* __restrict__ perm, const uint64_t* __restrict__ coff,
                       const uint64_t* __restrict__ ioff, const uint32_t* __restrict__ rank, const T* __restrict__ in,
                       T* __restrict__ out) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t i = warp; i < n; i += nwarps) {
    const uint64_t c0 = coff[perm[i]], i0 = ioff[i], len = ioff[i + 1] - i0;
    for (uint64_t k = lane; k < len; k += 32) {
      if (TO_INTERNAL) out[i0 + k] = in[c0 + rank[i0 + k]];
      else out[c0 + rank[i0 + k]] = in[i0 + k];
    }
  }
}

int map_ids(gre_graph g, std::vector<uint32_t>* ids, const char* what) {
  for (uint32_t& s : *ids) {
    if (s >= g->n) {
      set_error("%s: vertex %u >= n = %llu", what, s, (unsigned long long)g->n);
      return GRE_INVALID_ARG;
    }
    if (g->perm) s = g->h_iperm[s];
  }
  return GRE_SUCCESS;
}

int perm_out_begin(gre_graph g, void* out_dev, uint64_t rows, size_t elem, void** internal) {
  if (!g->perm) {
    *internal = out_dev;
    return GRE_SUCCESS;
  }
  return g->ws.get(WS_PERM_OUT, elem * rows * g->n, internal);
}

int perm_out_end(gre_graph g, const void* internal, void* out_dev, uint64_t rows, size_t elem) {
  if (!g->perm) return GRE_SUCCESS;
  const int grid = grid_for(rows * g->n, 256);
  if (elem == 4) k_unperm<uint32_t><<<grid, 256, 0, g->stream>>>(g->n, rows, g->iperm, (const uint32_t*)internal, (uint32_t*)out_dev);
  else if (elem == 8) k_unperm<uint64_t><<<grid, 256, 0, g->stream>>>(g->n, rows, g->iperm, (const uint64_t*)internal, (uint64_t*)out_dev);
  else return GRE_INVALID_ARG;
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

int perm_in(gre_graph g, const void* in_dev, size_t elem, int slot, const void** internal) {
  if (!g->perm || !in_dev) {
    *internal = in_dev;
    return GRE_SUCCESS;
  }
  void* p = nullptr;
  GRE_CHECK(g->ws.get(slot, elem * g->n, &p));
  const int grid = grid_for(g->n, 256);
  if (elem == 4) k_perm<uint32_t><<<grid, 256, 0, g->stream>>>(g->n, g->perm, (const uint32_t*)in_dev, (uint32_t*)p);
  else if (elem == 8) k_perm<uint64_t><<<grid, 256, 0, g->stream>>>(g->n, g->perm, (const uint64_t*)in_dev, (uint64_t*)p);
  else return GRE_INVALID_ARG;
  GRE_LAUNCH_CHECK();
  *internal = p;
  return GRE_SUCCESS;
}

// caller-order row offsets of the CSR (workspace slot WS_PERM_OFF)
static int caller_offsets(gre_graph g, uint64_t** coff) {
  const uint64_t n = g->n;
  void* p = nullptr;
  GRE_CHECK(g->ws.get(WS_PERM_OFF, sizeof(uint64_t) * 2 * (n + 1), &p));
  uint64_t* deg = (uint64_t*)p;
  uint64_t* off = deg + (n + 1);
  k_caller_degree<<<grid_for(n + 1, 256), 256, 0, g->stream>>>(n, g->iperm, g->off, deg);
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, deg, off, n + 1, g->stream);
  void* tmp = nullptr;
  GRE_CHECK(g->ws.get(WS_CUB, tb, &tmp));
  GRE_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, deg, off, n + 1, g->stream));
  *coff = off;
  return GRE_SUCCESS;
}

template <bool TO_INTERNAL>
static int arcs_move(gre_graph g, const void* in_dev, void* out_dev, size_t elem) {
  if (!g->perm) {
    if (in_dev != out_dev && g->m) GRE_CUDA(cudaMemcpyAsync(out_dev, in_dev, elem * g->m, cudaMemcpyDefault, g->stream));
    return GRE_SUCCESS;
  }
  uint64_t* coff = nullptr;
  GRE_CHECK(caller_offsets(g, &coff));
  const int grid = grid_for(g->n * 32, 256);
  if (elem == 4)
    k_arcs<uint32_t, TO_INTERNAL><<<grid, 256, 0, g->stream>>>(g->n, g->perm, coff, g->off, g->arc_rank, (const uint32_t*)in_dev,
                                                                      (uint32_t*)out_dev);
  else if (elem == 8)
    k_arcs<uint64_t, TO_INTERNAL><<<grid, 256, 0, g->stream>>>(g->n, g->perm, coff, g->off, g->arc_rank, (const uint64_t*)in_dev,
                                                                      (uint64_t*)out_dev);
  else return GRE_INVALID_ARG;
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

int arcs_to_internal(gre_graph g, const void* in_dev, void* out_dev, size_t elem) { return arcs_move<true>(g, in_dev, out_dev, elem); }
int arcs_to_caller(gre_graph g, const void* in_dev, void* out_dev, size_t elem) { return arcs_move<false>(g, in_dev, out_dev, elem); }

// Caller-order CSR: row offsets and neighbour ids of caller row v = internal row iperm[v].
__global__ void k_col_to_caller(uint64_t n, const uint32_t* __restrict__ perm, const uint64_t* __restrict__ coff,
                                const uint64_t* __restrict__ ioff, const uint32_t* __restrict__ rank, const uint32_t* __restrict__ icol,
                                uint32_t* __restrict__ out) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t i = warp; i < n; i += nwarps) {
    const uint64_t c0 = coff[perm[i]], i0 = ioff[i], len = ioff[i + 1] - i0;
    for (uint64_t k = lane; k < len; k += 32) out[c0 + rank[i0 + k]] = perm[icol[i0 + k]];
  }
}

int caller_csr(gre_graph g, uint64_t* off_out, uint32_t* col_out) {
  uint64_t* coff = nullptr;
  GRE_CHECK(caller_offsets(g, &coff));
  GRE_CUDA(cudaMemcpyAsync(off_out, coff, sizeof(uint64_t) * (g->n + 1), cudaMemcpyDefault, g->stream));
  if (g->m) {
    void* tmp = nullptr;
    uint32_t* dcol = col_out;
    if (!is_device_ptr(col_out)) {
      GRE_CHECK(g->ws.get(WS_PERM_OUT, sizeof(uint32_t) * g->m, &tmp));
      dcol = (uint32_t*)tmp;
    }
    k_col_to_caller<<<grid_for(g->n * 32, 256), 256, 0, g->stream>>>(g->n, g->perm, coff, g->off, g->arc_rank, g->col, dcol);
    GRE_LAUNCH_CHECK();
    if (dcol != col_out) GRE_CUDA(cudaMemcpyAsync(col_out, dcol, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost, g->stream));
  }
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  return GRE_SUCCESS;
}

}  // namespace gre
