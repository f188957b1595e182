// Betweenness centrality (Brandes), the reference's Forward/Backward plugins driven per source
// (Kernels/BC.hpp:56-163, usr/test_bc.cpp:63-110), accumulated bc(v) = sum_{s != v} dep_s(v).
//
// Per source the reference computes: forward, level and path count numPaths (sigma) by BFS
// with sum-combine; backward, one superstep per level i from the deepest down:
//   pathwgt[w] = (1 + dep[w]) / sigma[w] for w at level i, summed into each neighbour v,
//   dep[v] = sum[v] * sigma[v] for v at level i-1.
// Here both passes pull: a vertex v at level d adds, in its in-arc order, sigma[u] over
// neighbours u at level d-1 (forward) and (1 + dep[w]) / sigma[w] over neighbours w at level
// d+1 (backward).  Rows longer than 512 arcs are cut into fixed 512-arc chunks whose partial
// sums are added in chunk order.  Every per-(vertex, source) sum therefore has one association
// order, shared by:
//   * the single-source path (batched = 0): direction-optimising BFS levels, one thread per
//     vertex (or chunk) per level;
//   * the batched path (batched = 1): 64 sources per uint64 word.  A multi-source BFS stores the
//     frontier word F_d[v] of every level; a warp handles one vertex with lane j owning sources
//     j and j + 32; sigma and dep are [n][64] FP64 rows read 256 bytes per half-warp.
// so both produce bit-identical bc.  bc[v] adds dep_s(v) in source order in both.
//
// sigma is FP64 (the reference's int numPaths wraps beyond 2^31; the values agree below).
#include <algorithm>
#include <vector>

#include "gre_internal.cuh"
#include "msbfs.cuh"

namespace gre {

constexpr uint64_t kBcChunk = 512;

template <class T>
static int ws_array(gre_graph g, int slot, uint64_t count, T** p) {
  void* v = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &v));
  *p = (T*)v;
  return GRE_SUCCESS;
}

// The arithmetic of one arc term, written with explicit rounding so that both paths (and any
// compiler contraction setting) perform exactly the same operations.
__device__ __forceinline__ double dep_term(double dep_w, double sigma_w) { return __ddiv_rn(__dadd_rn(1.0, dep_w), sigma_w); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

static int ensure_bc_chunks(gre_graph g) {
  ChunkTable& T = g->bc_chunks;
  if (T.ready) return GRE_SUCCESS;
  const uint64_t n = g->n;
  std::vector<uint64_t> ho(n + 1);
  GRE_CUDA(cudaMemcpy(ho.data(), g->roff, sizeof(uint64_t) * (n + 1), cudaMemcpyDeviceToHost));
  std::vector<uint32_t> rows;
  std::vector<uint64_t> crow, cbeg, first;
  for (uint64_t v = 0; v < n; ++v) {
    if (ho[v + 1] - ho[v] <= kBcChunk) continue;
    first.push_back(crow.size());
    for (uint64_t a = ho[v]; a < ho[v + 1]; a += kBcChunk) {
      crow.push_back(rows.size());
      cbeg.push_back(a);
    }
    rows.push_back((uint32_t)v);
  }
  first.push_back(crow.size());
  T.ch = kBcChunk;
  T.nrows = rows.size();
  T.nchunks = crow.size();
  GRE_CUDA(cudaMalloc(&T.rows, sizeof(uint32_t) * (rows.size() + 1)));
  GRE_CUDA(cudaMalloc(&T.chunk_row, sizeof(uint64_t) * (crow.size() + 1)));
  GRE_CUDA(cudaMalloc(&T.chunk_begin, sizeof(uint64_t) * (cbeg.size() + 1)));
  GRE_CUDA(cudaMalloc(&T.first, sizeof(uint64_t) * first.size()));
  if (!rows.empty()) {
    GRE_CUDA(cudaMemcpy(T.rows, rows.data(), sizeof(uint32_t) * rows.size(), cudaMemcpyHostToDevice));
    GRE_CUDA(cudaMemcpy(T.chunk_row, crow.data(), sizeof(uint64_t) * crow.size(), cudaMemcpyHostToDevice));
    GRE_CUDA(cudaMemcpy(T.chunk_begin, cbeg.data(), sizeof(uint64_t) * cbeg.size(), cudaMemcpyHostToDevice));
  }
  GRE_CUDA(cudaMemcpy(T.first, first.data(), sizeof(uint64_t) * first.size(), cudaMemcpyHostToDevice));
  T.ready = true;
  return GRE_SUCCESS;
}

// ---------------------------------------------------------------------------------------------
// single source
// ---------------------------------------------------------------------------------------------
__global__ void k_level_hist(uint64_t n, const int32_t* __restrict__ level, uint32_t* __restrict__ hist) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t l = level[v];
    if (l >= 0) atomicAdd(hist + l, 1u);
  }
}
__global__ void k_level_scatter(uint64_t n, const int32_t* __restrict__ level, uint32_t* __restrict__ cursor, uint32_t* __restrict__ list) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t l = level[v];
    if (l >= 0) list[atomicAdd(cursor + l, 1u)] = (uint32_t)v;
  }
}

struct Bc1 {
  const uint64_t* __restrict__ roff;
  const uint32_t* __restrict__ rcol;
  const int32_t* __restrict__ level;
  double* sigma;
  double* dep;
  // sum over arcs [a0, a1) of the forward (sigma) or backward (dep) term for level d
  __device__ __forceinline__ double fwd(uint64_t a0, uint64_t a1, int32_t d) const {
    double acc = 0.0;
    for (uint64_t a = a0; a < a1; ++a) {
      const uint32_t u = __ldg(rcol + a);
      if (level[u] == d - 1) acc = add(acc, sigma[u]);
    }
    return acc;
  }
  __device__ __forceinline__ double bwd(uint64_t a0, uint64_t a1, int32_t d) const {
    double acc = 0.0;
    for (uint64_t a = a0; a < a1; ++a) {
      const uint32_t w = __ldg(rcol + a);
      if (level[w] == d + 1) acc = add(acc, dep_term(dep[w], sigma[w]));
    }
    return acc;
  }
};

template <bool FWD>
__global__ void k_bc1_rows(const uint32_t* __restrict__ list, uint64_t cnt, int32_t d, Bc1 B, uint64_t ch) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = list[i];
    const uint64_t a0 = B.roff[v], a1 = B.roff[v + 1];
    if (a1 - a0 > ch) continue;  // chunked
    if (FWD) B.sigma[v] = B.fwd(a0, a1, d);
    else B.dep[v] = __dmul_rn(B.sigma[v], B.bwd(a0, a1, d));
  }
}

template <bool FWD>
__global__ void k_bc1_chunks(ChunkTable T, int32_t d, Bc1 B, double* __restrict__ partial) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < T.nchunks; c += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = T.rows[T.chunk_row[c]];
    if (B.level[v] != d) continue;
    const uint64_t a0 = T.chunk_begin[c];
    const uint64_t end = B.roff[v + 1];
    const uint64_t a1 = a0 + T.ch < end ? a0 + T.ch : end;
    partial[c] = FWD ? B.fwd(a0, a1, d) : B.bwd(a0, a1, d);
  }
}

template <bool FWD>
__global__ void k_bc1_finish(ChunkTable T, int32_t d, Bc1 B, const double* __restrict__ partial) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < T.nrows; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = T.rows[i];
    if (B.level[v] != d) continue;
    double s = 0.0;
    for (uint64_t c = T.first[i]; c < T.first[i + 1]; ++c) s = add(s, partial[c]);
    if (FWD) B.sigma[v] = s;
    else B.dep[v] = __dmul_rn(B.sigma[v], s);
  }
}

__global__ void k_bc1_init(uint64_t n, uint32_t s, double* __restrict__ sigma, double* __restrict__ dep) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    sigma[v] = (v == s) ? 1.0 : 0.0;
    dep[v] = 0.0;
  }
}

__global__ void k_bc1_accumulate(uint64_t n, uint32_t s, const double* __restrict__ dep, double* __restrict__ bc) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    if (v != s) bc[v] = add(bc[v], dep[v]);
}

static int bc_single(gre_graph g, const std::vector<uint32_t>& hs, double* dbc, gre_stats* st) {
  const uint64_t n = g->n;
  const ChunkTable& T = g->bc_chunks;
  int32_t* level;
  double *sigma, *dep, *partial;
  uint32_t *list, *hist, *roots;
  GRE_CHECK(ws_array(g, WS_BC0, n, &level));
  GRE_CHECK(ws_array(g, WS_BC1, n, &sigma));
  GRE_CHECK(ws_array(g, WS_BC2, n, &dep));
  GRE_CHECK(ws_array(g, WS_BC3, n, &list));
  GRE_CHECK(ws_array(g, WS_BC5, T.nchunks + 1, &partial));
  GRE_CHECK(ws_array(g, WS_BC7, hs.size() + 1, &roots));
  GRE_CUDA(cudaMemcpyAsync(roots, hs.data(), sizeof(uint32_t) * hs.size(), cudaMemcpyHostToDevice, g->stream));
  uint64_t arcs = 0, bytes = 0;
  for (size_t i = 0; i < hs.size(); ++i) {
    const uint32_t s = hs[i];
    GRE_CHECK(bfs_levels(g, roots + i, 1, level, nullptr, false));
    // vertices grouped by level
    uint32_t nl = 0;
    {
      int32_t maxl = 0;
      // levels fit below n; a histogram of n+1 bins is enough
      GRE_CHECK(ws_array(g, WS_BC4, n + 2, &hist));
      GRE_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (n + 2), g->stream));
      k_level_hist<<<grid_for(n, 256), 256, 0, g->stream>>>(n, level, hist);
      // BFS levels are contiguous from 0, so the first empty bin ends them; the bins are read
      // back in growing blocks until one holds an empty bin (one 16 KB read for most graphs)
      std::vector<uint32_t> hh;
      uint64_t have = 0;
      maxl = -1;
      while (maxl < 0 && have < n + 2) {
        const uint64_t take = std::min<uint64_t>(n + 2 - have, std::max<uint64_t>(4096, have));
        hh.resize(have + take);
        GRE_CUDA(cudaMemcpyAsync(hh.data() + have, hist + have, sizeof(uint32_t) * take, cudaMemcpyDeviceToHost,
                                 g->stream));
        GRE_CUDA(cudaStreamSynchronize(g->stream));
        uint64_t l = have;
        while (l < have + take && hh[l]) ++l;
        if (l < have + take) maxl = (int32_t)l - 1;
        have += take;
      }
      nl = (uint32_t)maxl + 1;
      std::vector<uint32_t> start(nl + 1, 0);
      for (uint32_t l = 0; l < nl; ++l) start[l + 1] = start[l] + hh[l];
      GRE_CUDA(cudaMemcpyAsync(hist, start.data(), sizeof(uint32_t) * nl, cudaMemcpyHostToDevice, g->stream));
      k_level_scatter<<<grid_for(n, 256), 256, 0, g->stream>>>(n, level, hist, list);
      k_bc1_init<<<grid_for(n, 256), 256, 0, g->stream>>>(n, s, sigma, dep);
      GRE_LAUNCH_CHECK();
      Bc1 B{g->roff, g->rcol, level, sigma, dep};
      for (int32_t d = 1; d < (int32_t)nl; ++d) {
        const uint64_t cnt = hh[d];
        k_bc1_rows<true><<<grid_for(cnt, 128, 8), 128, 0, g->stream>>>(list + start[d], cnt, d, B, T.ch);
        if (T.nchunks) {
          k_bc1_chunks<true><<<grid_for(T.nchunks, 128, 8), 128, 0, g->stream>>>(T, d, B, partial);
          k_bc1_finish<true><<<grid_for(T.nrows, 128, 4), 128, 0, g->stream>>>(T, d, B, partial);
        }
      }
      for (int32_t d = (int32_t)nl - 2; d >= 0; --d) {
        const uint64_t cnt = hh[d];
        k_bc1_rows<false><<<grid_for(cnt, 128, 8), 128, 0, g->stream>>>(list + start[d], cnt, d, B, T.ch);
        if (T.nchunks) {
          k_bc1_chunks<false><<<grid_for(T.nchunks, 128, 8), 128, 0, g->stream>>>(T, d, B, partial);
          k_bc1_finish<false><<<grid_for(T.nrows, 128, 4), 128, 0, g->stream>>>(T, d, B, partial);
        }
      }
      k_bc1_accumulate<<<grid_for(n, 256), 256, 0, g->stream>>>(n, s, dep, dbc);
      GRE_LAUNCH_CHECK();
    }
    arcs += 2 * g->m;
    bytes += 2 * (8 * (n + 1) + 4 * g->m) + 24 * n;
    if (st) st->supersteps += 2 * nl;
  }
  if (st) {
    st->arcs_traversed += arcs;
    st->algo_bytes += bytes;
  }
  return GRE_SUCCESS;
}

// ---------------------------------------------------------------------------------------------
// batched: 64 sources per word
// ---------------------------------------------------------------------------------------------
__global__ void k_bcm_seed(const uint32_t* __restrict__ srcs, uint32_t k, unsigned long long* __restrict__ seen,
                           unsigned long long* __restrict__ f0, double* __restrict__ sigma) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (uint32_t j = 0; j < k; ++j) {
    const uint32_t s = srcs[j];
    seen[s] |= 1ull << j;
    f0[s] |= 1ull << j;
    sigma[(uint64_t)s * 64 + j] = 1.0;
  }
}

// F_next[v] = (OR over in-neighbours u of F_d[u]) & ~seen[v]; early exit when all unseen found
__global__ void __launch_bounds__(256) k_bcm_forward(uint64_t n, unsigned long long full, const uint64_t* __restrict__ roff,
                                                     const uint32_t* __restrict__ rcol, const unsigned long long* __restrict__ fd,
                                                     unsigned long long* __restrict__ fnext, unsigned long long* __restrict__ seen,
                                                     unsigned long long* __restrict__ counters) {
  unsigned long long found = 0, scanned = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long s = seen[v];
    const unsigned long long want = full & ~s;
    unsigned long long nb = 0;
    if (want) {
      unsigned long long acc = 0;
      const uint64_t a1 = roff[v + 1];
      for (uint64_t a = roff[v]; a < a1; ++a) {
        acc |= fd[__ldg(rcol + a)];
        ++scanned;
        if ((acc & want) == want) break;
      }
      nb = acc & want;
      if (nb) seen[v] = s | nb;
    }
    fnext[v] = nb;
    found += nb != 0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    found += __shfl_xor_sync(0xffffffffu, found, o);
    scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
  }
  if ((threadIdx.x & 31u) == 0) {
    if (found) atomicAdd(counters, found);
    if (scanned) atomicAdd(counters + 1, scanned);
  }
}

// list of vertices with a non-zero frontier word
__global__ void k_bcm_list(uint64_t n, const unsigned long long* __restrict__ f, uint32_t* __restrict__ list,
                           unsigned int* __restrict__ count) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < n; base += stride) {
    const uint64_t v = base + (threadIdx.x & 31u);
    const bool nz = v < n && f[v] != 0;
    const uint32_t pos = warp_append(count, nz);
    if (nz) list[pos] = (uint32_t)v;
  }
}

struct BcM {
  const uint64_t* __restrict__ roff;
  const uint32_t* __restrict__ rcol;
  const unsigned long long* __restrict__ fprev;  // F_{d-1} (forward) or F_{d+1} (backward)
  const unsigned long long* __restrict__ fd;     // F_d
  double* sigma;                                 // [n][64]
  double* dep;                                   // [n][64]
  // Arcs [a0, a1) of vertex v; lane owns sources lane and lane+32.  32 arcs at a time are staged
  // with lane = arc (column and source mask loaded 32-wide), compacted to the arcs whose mask
  // meets v's, then walked in arc order with lane = source: the same association order as one
  // source at a time, with the index and mask loads off the per-arc critical path.
  // su / sm: this warp's 32-entry shared-memory staging area.
  template <bool FWD>
  __device__ __forceinline__ void sum(uint32_t v, uint64_t a0, uint64_t a1, double& acc0, double& acc1, uint32_t* su,
                                      unsigned long long* sm) const {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long mine = fd[v];
    for (uint64_t base = a0; base < a1; base += 32) {
      const uint64_t a = base + lane;
      uint32_t u = 0;
      unsigned long long m = 0;
      if (a < a1) {
        u = __ldg(rcol + a);
        m = fprev[u] & mine;
      }
      const uint32_t ball = __ballot_sync(0xffffffffu, m != 0ull);
      if (m) {
        const uint32_t pos = __popc(ball & ((1u << lane) - 1u));
        su[pos] = u;
        sm[pos] = m;
      }
      __syncwarp();
      const int cnt = __popc(ball);
#pragma unroll 4
      for (int i = 0; i < cnt; ++i) {
        const uint64_t row = (uint64_t)su[i] * 64;
        const unsigned long long mm = sm[i];
        // forward: sigma holds path counts; backward: the children's entries already hold their
        // pull weights dep_term(dep, sigma) (k_bcm_weights), the same value the looped path
        // computes per arc
        if ((mm >> lane) & 1ull) acc0 = add(acc0, sigma[row + lane]);
        if ((mm >> (lane + 32)) & 1ull) acc1 = add(acc1, sigma[row + lane + 32]);
      }
      __syncwarp();
    }
  }
  template <bool FWD>
  __device__ __forceinline__ void store(uint32_t v, double acc0, double acc1) const {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long mine = fd[v];
    const uint64_t row = (uint64_t)v * 64;
    if ((mine >> lane) & 1ull) {
      if (FWD) sigma[row + lane] = acc0;
      else dep[row + lane] = __dmul_rn(sigma[row + lane], acc0);
    }
    if ((mine >> (lane + 32)) & 1ull) {
      if (FWD) sigma[row + lane + 32] = acc1;
      else dep[row + lane + 32] = __dmul_rn(sigma[row + lane + 32], acc1);
    }
  }
};

// Backward: once the dependencies of a level are final, each of its (vertex, source) entries of
// sigma is replaced by the weight its parents pull, dep_term(dep, sigma) = (1 + dep) / sigma:
// one division per entry instead of one per arc and source, and one load per term instead of
// two.  The entry's sigma is not read again (its own dependency is already stored).
__global__ void __launch_bounds__(256) k_bcm_weights(const uint32_t* __restrict__ list, const unsigned int* __restrict__ count,
                                                     const unsigned long long* __restrict__ F, double* __restrict__ sigma,
                                                     const double* __restrict__ dep) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t cnt = *count;
  for (uint64_t i = warp; i < cnt; i += nwarps) {
    const uint32_t w = list[i];
    const unsigned long long word = F[w];
    const uint64_t row = (uint64_t)w * 64;
    if ((word >> lane) & 1ull) sigma[row + lane] = dep_term(dep[row + lane], sigma[row + lane]);
    if ((word >> (lane + 32)) & 1ull) sigma[row + lane + 32] = dep_term(dep[row + lane + 32], sigma[row + lane + 32]);
  }
}

template <bool FWD>
__global__ void __launch_bounds__(256) k_bcm_rows(const uint32_t* __restrict__ list, const unsigned int* __restrict__ count, BcM B,
                                                  uint64_t ch) {
  __shared__ uint32_t s_u[8][32];
  __shared__ unsigned long long s_m[8][32];
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t cnt = *count;
  for (uint64_t i = warp; i < cnt; i += nwarps) {
    const uint32_t v = list[i];
    const uint64_t a0 = B.roff[v], a1 = B.roff[v + 1];
    if (a1 - a0 > ch) continue;
    double acc0 = 0.0, acc1 = 0.0;
    B.template sum<FWD>(v, a0, a1, acc0, acc1, s_u[threadIdx.x >> 5], s_m[threadIdx.x >> 5]);
    B.template store<FWD>(v, acc0, acc1);
  }
}

template <bool FWD>
__global__ void __launch_bounds__(256) k_bcm_chunks(ChunkTable T, BcM B, double* __restrict__ partial) {
  __shared__ uint32_t s_u[8][32];
  __shared__ unsigned long long s_m[8][32];
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t c = warp; c < T.nchunks; c += nwarps) {
    const uint32_t v = T.rows[T.chunk_row[c]];
    if (!B.fd[v]) continue;
    const uint64_t a0 = T.chunk_begin[c];
    const uint64_t end = B.roff[v + 1];
    const uint64_t a1 = a0 + T.ch < end ? a0 + T.ch : end;
    double acc0 = 0.0, acc1 = 0.0;
    B.template sum<FWD>(v, a0, a1, acc0, acc1, s_u[threadIdx.x >> 5], s_m[threadIdx.x >> 5]);
    partial[c * 64 + lane] = acc0;
    partial[c * 64 + lane + 32] = acc1;
  }
}

template <bool FWD>
__global__ void __launch_bounds__(256) k_bcm_finish(ChunkTable T, BcM B, const double* __restrict__ partial) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t i = warp; i < T.nrows; i += nwarps) {
    const uint32_t v = T.rows[i];
    if (!B.fd[v]) continue;
    double s0 = 0.0, s1 = 0.0;
    for (uint64_t c = T.first[i]; c < T.first[i + 1]; ++c) {
      s0 = add(s0, partial[c * 64 + lane]);
      s1 = add(s1, partial[c * 64 + lane + 32]);
    }
    B.template store<FWD>(v, s0, s1);
  }
}

__global__ void k_bcm_accumulate(uint64_t n, const uint32_t* __restrict__ srcs, uint32_t k, const double* __restrict__ dep,
                                 double* __restrict__ bc) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    double b = bc[v];
    for (uint32_t j = 0; j < k; ++j)
      if (srcs[j] != v) b = add(b, dep[v * 64 + j]);
    bc[v] = b;
  }
}

static int fpool_levels(gre_graph g, uint64_t levels) {
  if (g->bc_fpool_levels >= levels) return GRE_SUCCESS;
  uint64_t want = std::max<uint64_t>(levels, std::max<uint64_t>(32, 2 * g->bc_fpool_levels));
  uint64_t* p = nullptr;
  GRE_CUDA(cudaMalloc(&p, sizeof(uint64_t) * g->n * want));
  if (g->bc_fpool) {
    GRE_CUDA(cudaMemcpyAsync(p, g->bc_fpool, sizeof(uint64_t) * g->n * g->bc_fpool_levels, cudaMemcpyDeviceToDevice, g->stream));
    GRE_CUDA(cudaStreamSynchronize(g->stream));
    cudaFree(g->bc_fpool);
  }
  g->bc_fpool = p;
  g->bc_fpool_levels = want;
  return GRE_SUCCESS;
}

static int bc_batched(gre_graph g, const std::vector<uint32_t>& hs, double* dbc, gre_stats* st) {
  const uint64_t n = g->n;
  const ChunkTable& T = g->bc_chunks;
  double *sigma, *dep, *partial;
  uint32_t *list, *srcs;
  unsigned long long *seen, *cnt, *acc;
  GRE_CHECK(ws_array(g, WS_BC1, n * 64, &sigma));
  GRE_CHECK(ws_array(g, WS_BC2, n * 64, &dep));
  GRE_CHECK(ws_array(g, WS_BC3, n, &list));
  GRE_CHECK(ws_array(g, WS_BC4, n, &seen));
  GRE_CHECK(ws_array(g, WS_BC5, (T.nchunks + 1) * 64, &partial));
  GRE_CHECK(ws_array(g, WS_BC6, 8, &cnt));
  GRE_CHECK(ensure_bins(g, true));
  GRE_CHECK(ws_array(g, WS_BC0, n, &acc));
  GRE_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * n, g->stream));
  GRE_CHECK(ws_array(g, WS_BC7, 64, &srcs));
  GRE_CHECK(fpool_levels(g, 32));
  uint64_t arcs = 0, bytes = 0;
  const int sms = num_sms();
  for (size_t j0 = 0; j0 < hs.size(); j0 += 64) {
    const uint32_t k = (uint32_t)std::min<size_t>(64, hs.size() - j0);
    const unsigned long long full = k == 64 ? ~0ull : ((1ull << k) - 1ull);
    GRE_CUDA(cudaMemcpyAsync(srcs, hs.data() + j0, sizeof(uint32_t) * k, cudaMemcpyHostToDevice, g->stream));
    GRE_CUDA(cudaMemsetAsync(sigma, 0, sizeof(double) * n * 64, g->stream));
    GRE_CUDA(cudaMemsetAsync(dep, 0, sizeof(double) * n * 64, g->stream));
    GRE_CUDA(cudaMemsetAsync(seen, 0, sizeof(unsigned long long) * n, g->stream));
    GRE_CUDA(cudaMemsetAsync(g->bc_fpool, 0, sizeof(unsigned long long) * n, g->stream));
    k_bcm_seed<<<1, 32, 0, g->stream>>>(srcs, k, seen, (unsigned long long*)g->bc_fpool, sigma);
    // forward: frontier words of every level
    uint64_t nl = 1;  // levels stored: F_0 .. F_{nl-1}
    unsigned long long live = full;  // sources whose frontier is not empty
    while (true) {
      GRE_CHECK(fpool_levels(g, nl + 1));
      unsigned long long* fd = (unsigned long long*)g->bc_fpool + (nl - 1) * n;
      unsigned long long* fn = (unsigned long long*)g->bc_fpool + nl * n;
      // push from a sparse frontier, pull otherwise (same frontier words either way)
      GRE_CUDA(cudaMemsetAsync(cnt, 0, 64, g->stream));
      ms::k_frontier_list<<<grid_for(n, 256, 8), 256, 0, g->stream>>>(n, fd, g->off, list, (unsigned int*)(cnt + 2), cnt + 3);
      unsigned long long h[6];
      GRE_CUDA(cudaMemcpyAsync(h, cnt, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      const bool push = h[3] * 14 < g->m;
      if (push)
        ms::k_push<<<grid_for((h[2] & 0xffffffffull) * 32, 256, 8), 256, 0, g->stream>>>(list, (unsigned int*)(cnt + 2), g->off,
                                                                                          g->col, fd, seen, acc);
      else
        GRE_CHECK(ms::pull(g->bins_in, live, g->roff, g->rcol, fd, seen, acc, cnt + 4, g->stream));
      ms::k_commit<<<grid_for(n, 256, 8), 256, 0, g->stream>>>(n, acc, seen, fn, nullptr, 0, cnt, cnt + 5);
      GRE_LAUNCH_CHECK();
      GRE_CUDA(cudaMemcpyAsync(h, cnt, sizeof h, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      if (push) {
        arcs += h[3];
        bytes += 16 * (h[2] & 0xffffffffull) + 12 * h[3] + 32 * n;
      } else {
        arcs += h[4];
        bytes += 24 * n + 12 * h[4];
      }
      if (h[0] == 0) break;
      live = h[5];
      ++nl;
    }
    unsigned long long* F = (unsigned long long*)g->bc_fpool;
    auto level_pass = [&](bool fwd, uint64_t d) -> int {
      BcM B{g->roff, g->rcol, fwd ? F + (d - 1) * n : F + (d + 1) * n, F + d * n, sigma, dep};
      // backward: `list` still holds F_{d+1} (built by the previous pass: the last forward pass
      // for the deepest level), whose dependencies are final
      if (!fwd) k_bcm_weights<<<sms * 8, 256, 0, g->stream>>>(list, (unsigned int*)cnt, F + (d + 1) * n, sigma, dep);
      GRE_CUDA(cudaMemsetAsync(cnt, 0, 4, g->stream));
      k_bcm_list<<<grid_for(n, 256, 8), 256, 0, g->stream>>>(n, F + d * n, list, (unsigned int*)cnt);
      const int grid = sms * 8;
      if (fwd) {
        k_bcm_rows<true><<<grid, 256, 0, g->stream>>>(list, (unsigned int*)cnt, B, T.ch);
        if (T.nchunks) {
          k_bcm_chunks<true><<<grid_for(T.nchunks * 32, 256, 8), 256, 0, g->stream>>>(T, B, partial);
          k_bcm_finish<true><<<grid_for(T.nrows * 32, 256, 4), 256, 0, g->stream>>>(T, B, partial);
        }
      } else {
        k_bcm_rows<false><<<grid, 256, 0, g->stream>>>(list, (unsigned int*)cnt, B, T.ch);
        if (T.nchunks) {
          k_bcm_chunks<false><<<grid_for(T.nchunks * 32, 256, 8), 256, 0, g->stream>>>(T, B, partial);
          k_bcm_finish<false><<<grid_for(T.nrows * 32, 256, 4), 256, 0, g->stream>>>(T, B, partial);
        }
      }
      GRE_LAUNCH_CHECK();
      return GRE_SUCCESS;
    };
    // levels 1 .. nl-1 hold vertices (F_{nl} is empty)
    for (uint64_t d = 1; d < nl; ++d) GRE_CHECK(level_pass(true, d));
    for (int64_t d = (int64_t)nl - 2; d >= 0; --d) GRE_CHECK(level_pass(false, (uint64_t)d));
    k_bcm_accumulate<<<grid_for(n, 256), 256, 0, g->stream>>>(n, srcs, k, dep, dbc);
    GRE_LAUNCH_CHECK();
    arcs += 2 * g->m;
    bytes += 2 * nl * 8 * n + 2 * (8 * (n + 1) + 12 * g->m) + 2 * 512 * (uint64_t)n;
    if (st) st->supersteps += (uint32_t)(2 * nl);
  }
  if (st) {
    st->arcs_traversed += arcs;
    st->algo_bytes += bytes;
  }
  return GRE_SUCCESS;
}

}  // namespace gre

using namespace gre;

extern "C" {

int gre_bc(gre_graph g, const uint32_t* srcs, uint32_t nsrc, int batched, double* bc, gre_stats* st) {
  if (!g || !bc || (nsrc && !srcs)) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  std::vector<uint32_t> hs(nsrc);
  if (nsrc) GRE_CUDA(cudaMemcpy(hs.data(), srcs, sizeof(uint32_t) * nsrc, cudaMemcpyDefault));
  GRE_CHECK(map_ids(g, &hs, "gre_bc"));
  GRE_CHECK(ensure_bc_chunks(g));
  double *dfinal, *dbc;
  GRE_CHECK(prepare_output(g, bc, n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, 1, 8, (void**)&dbc));
  RunTimer timer(g);
  GRE_CUDA(cudaMemsetAsync(dbc, 0, sizeof(double) * n, g->stream));
  if (batched) GRE_CHECK(bc_batched(g, hs, dbc, st));
  else GRE_CHECK(bc_single(g, hs, dbc, st));
  GRE_CHECK(perm_out_end(g, dbc, dfinal, 1, 8));
  GRE_CHECK(finish_output(g, bc, dfinal, n));
  GRE_CHECK(timer.stop(st));
  if (st) st->traversed_edges = (uint64_t)nsrc * (g->symmetric() ? g->m / 2 : g->m);
  return GRE_SUCCESS;
}

}  // extern "C"
