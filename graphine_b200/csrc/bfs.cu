// BFS fast paths.
//
// The reference BFS (Kernels/BFS.hpp:34-72 on Engine.hpp's superstep) expands every frontier
// vertex over its arcs, claims unvisited neighbours first-writer-wins under a lock and makes
// them the next frontier; levels are the superstep of discovery.  Here:
//
//  * gre_bfs / gre_bfs_multiroot: direction-optimising BFS (Beamer, Asanovic, Patterson 2012).
//    Top-down steps expand a frontier queue edge-balanced: one thread per frontier arc, the
//    owning vertex found by binary search in the exclusive scan of frontier degrees; a visited
//    bitmap (n/8 bytes, L2-resident) filters claims, atomicOr claims a vertex.  Bottom-up steps
//    give each unvisited vertex one thread that scans its in-arcs for a parent in the frontier
//    bitmap and stops at the first; a warp covers 32 consecutive vertices, so the next-frontier
//    word is one __ballot_sync and needs no atomics.  Switch rule: to bottom-up when the
//    frontier's arcs exceed (unvisited arcs)/15, back to top-down when the frontier holds fewer
//    than n/18 vertices.
//  * gre_msbfs: 64 sources per uint64 word (multi-source BFS, Then et al. 2014): seen/frontier
//    words per vertex; a level is one pull over in-arcs OR-ing neighbour frontier words, so the
//    topology is read once per level for all 64 sources.
//
// Byte model, top-down level: 16 F (queue + offsets) + 8 A (column + visited probe) + 8 N;
// bottom-up level: 16 U (offsets + level of unvisited) + 4.125 A (column + frontier bit) + 4 N
// + n/8 (bitmap).  F frontier, A arcs scanned, U unvisited vertices scanned, N newly visited.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>

#include "gre_internal.cuh"
#include "msbfs.cuh"

namespace gre {

// persist.cu
bool msbfs_persistent_available(uint64_t n);
size_t msbfs_ctl_bytes();
int msbfs_word_persistent(gre_graph g, unsigned long long full, unsigned long long* seen, unsigned long long* fa,
                          unsigned long long* fb, unsigned long long* acc, uint32_t* list0, uint32_t* list1, int32_t* levels,
                          void* ctl_mem, unsigned long long* found_per_level, uint32_t* levels_out, uint64_t* scanned,
                          uint64_t* bytes, std::vector<unsigned long long>* found);

template <class T>
static int ws_array(gre_graph g, int slot, uint64_t count, T** p) {
  void* v = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &v));
  *p = (T*)v;
  return GRE_SUCCESS;
}

struct BfsCounters {
  unsigned long long next_count;  // vertices discovered in this level
  unsigned long long next_arcs;   // sum of their (out) degrees
  unsigned long long scanned;     // arcs scanned in this level
  unsigned long long pad;
};

__global__ void k_bfs_seed(const uint32_t* __restrict__ roots, uint32_t nroots, int32_t* __restrict__ level,
                           uint32_t* __restrict__ vis, uint32_t* __restrict__ queue, const uint64_t* __restrict__ off,
                           BfsCounters* __restrict__ c) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t q = 0;
  unsigned long long arcs = 0;
  for (uint32_t i = 0; i < nroots; ++i) {
    const uint32_t r = roots[i];
    if (vis[r >> 5] & (1u << (r & 31u))) continue;
    vis[r >> 5] |= 1u << (r & 31u);
    level[r] = 0;
    queue[q++] = r;
    arcs += off[r + 1] - off[r];
  }
  c->next_count = q;
  c->next_arcs = arcs;
}

__global__ void k_frontier_degrees(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ off,
                                   uint64_t* __restrict__ deg) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = queue[i];
    deg[i] = off[u + 1] - off[u];
  }
}

// One thread per frontier arc; prefix = exclusive scan of frontier degrees.
__global__ void __launch_bounds__(256) k_td_expand(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ prefix,
                                                   uint64_t total, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                   uint32_t* __restrict__ vis, int32_t* __restrict__ level, int32_t next_level,
                                                   uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ c) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  // iterate warp-uniformly so warp_append sees all 32 lanes
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < total; base += stride) {
    const uint64_t t = base + (threadIdx.x & 31u);
    bool claim = false;
    uint32_t v = 0;
    unsigned long long dv = 0;
    if (t < total) {
      // largest i with prefix[i] <= t
      uint64_t lo = 0, hi = nq;
      while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= t) lo = mid;
        else hi = mid;
      }
      const uint32_t u = queue[lo];
      v = __ldg(col + off[u] + (t - prefix[lo]));
      const uint32_t bit = 1u << (v & 31u);
      if (!(vis[v >> 5] & bit)) {
        const uint32_t old = atomicOr(vis + (v >> 5), bit);
        if (!(old & bit)) {
          claim = true;
          level[v] = next_level;
          dv = off[v + 1] - off[v];
        }
      }
    }
    const uint32_t pos = warp_append((uint32_t*)&c->pad, claim);  // slot counter lives in pad
    if (claim) next_queue[pos] = v;
    unsigned long long s = dv;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31u) == 0 && s) atomicAdd(&c->next_arcs, s);
  }
}

__global__ void k_queue_to_bits(const uint32_t* __restrict__ queue, uint64_t nq, uint32_t* __restrict__ bits) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = queue[i];
    atomicOr(bits + (v >> 5), 1u << (v & 31u));
  }
}

// Bottom-up level over in-arcs (roff/rcol); warp = one 32-vertex bitmap word.
__global__ void __launch_bounds__(256) k_bu_step(uint64_t n, const uint64_t* __restrict__ roff, const uint32_t* __restrict__ rcol,
                                                 const uint64_t* __restrict__ off, const uint32_t* __restrict__ front,
                                                 uint32_t* __restrict__ next, uint32_t* __restrict__ vis, int32_t* __restrict__ level,
                                                 int32_t next_level, BfsCounters* __restrict__ c) {
  const uint64_t nwords = (n + 31) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long found_arcs = 0, scanned = 0, found_n = 0;
  for (uint64_t w = warp; w < nwords; w += nwarps) {
    const uint32_t vw = vis[w];
    if (vw == 0xffffffffu) {
      if (lane == 0) next[w] = 0;
      continue;
    }
    const uint64_t v = (w << 5) + lane;
    bool found = false;
    if (v < n && !((vw >> lane) & 1u)) {
      const uint64_t a1 = roff[v + 1];
      for (uint64_t a = roff[v]; a < a1; ++a) {
        const uint32_t u = __ldg(rcol + a);
        ++scanned;
        if ((__ldg(front + (u >> 5)) >> (u & 31u)) & 1u) {
          found = true;
          break;
        }
      }
      if (found) {
        level[v] = next_level;
        found_arcs += off[v + 1] - off[v];
        ++found_n;
      }
    }
    const uint32_t ball = __ballot_sync(0xffffffffu, found);
    if (lane == 0) {
      next[w] = ball;
      if (ball) vis[w] = vw | ball;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    found_arcs += __shfl_xor_sync(0xffffffffu, found_arcs, o);
    scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
    found_n += __shfl_xor_sync(0xffffffffu, found_n, o);
  }
  if (lane == 0) {
    if (found_n) atomicAdd(&c->next_count, found_n);
    if (found_arcs) atomicAdd(&c->next_arcs, found_arcs);
    if (scanned) atomicAdd(&c->scanned, scanned);
  }
}

// bitmap -> queue (order within a warp's 32 words is by vertex id)
__global__ void k_bits_to_queue(uint64_t n, const uint32_t* __restrict__ bits, uint32_t* __restrict__ queue,
                                unsigned long long* __restrict__ count) {
  const uint64_t nwords = (n + 31) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = tid - lane; base < nwords; base += nthreads) {
    const uint64_t w = base + lane;
    const uint32_t word = (w < nwords) ? bits[w] : 0u;
    const uint32_t cnt = __popc(word);
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long pos = 0;
    if (lane == 31 && total) pos = atomicAdd(count, (unsigned long long)total);
    pos = __shfl_sync(0xffffffffu, pos, 31) + incl - cnt;
    uint32_t x = word;
    while (x) {
      const uint32_t b = __ffs(x) - 1;
      x &= x - 1;
      queue[pos++] = (uint32_t)(w << 5) + b;
    }
  }
}

// One direction-optimising BFS from `roots`, levels written into `level` (n int32).
int bfs_levels(gre_graph g, const uint32_t* droots, uint32_t nroots, int32_t* level, gre_stats* st, bool record) {
  const uint64_t n = g->n, m = g->m;
  const uint64_t nwords = (n + 31) >> 5;
  uint32_t *vis, *qa, *qb, *bits_a, *bits_b;
  uint64_t *deg, *prefix;
  BfsCounters* c;
  GRE_CHECK(ws_array(g, WS_A, nwords, &vis));
  GRE_CHECK(ws_array(g, WS_B, n, &qa));
  GRE_CHECK(ws_array(g, WS_C, n, &qb));
  GRE_CHECK(ws_array(g, WS_D, nwords, &bits_a));
  GRE_CHECK(ws_array(g, WS_E, nwords, &bits_b));
  GRE_CHECK(ws_array(g, WS_F, n + 1, &deg));
  GRE_CHECK(ws_array(g, WS_G, n + 1, &prefix));
  GRE_CHECK(ws_array(g, WS_COUNTERS, 4, &c));
  void* cubtmp = nullptr;
  size_t cubbytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cubbytes, deg, prefix, n + 1, g->stream);
  GRE_CHECK(g->ws.get(WS_CUB, cubbytes, &cubtmp));

  GRE_CUDA(cudaMemsetAsync(level, 0xff, sizeof(int32_t) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(vis, 0, sizeof(uint32_t) * nwords, g->stream));
  GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), g->stream));
  k_bfs_seed<<<1, 32, 0, g->stream>>>(droots, nroots, level, vis, qa, g->off, c);
  BfsCounters h;
  GRE_CUDA(cudaMemcpyAsync(&h, c, sizeof h, cudaMemcpyDeviceToHost, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  uint64_t nf = h.next_count, mf = h.next_arcs;
  int64_t mu = (int64_t)m - (int64_t)mf;
  bool bottom_up = false;
  uint32_t* queue = qa;
  uint32_t* nqueue = qb;
  uint32_t* front = bits_a;
  uint32_t* nbits = bits_b;
  int32_t d = 0;
  uint64_t scanned_total = 0, bytes = 0, visited = nf;
  const int sms = num_sms();
  while (nf > 0) {
    // direction choice
    if (!bottom_up && (double)mf > (double)mu / 15.0 && nf > 64) {
      GRE_CUDA(cudaMemsetAsync(front, 0, sizeof(uint32_t) * nwords, g->stream));
      k_queue_to_bits<<<grid_for(nf, 256), 256, 0, g->stream>>>(queue, nf, front);
      bottom_up = true;
    } else if (bottom_up && nf < n / 18) {
      GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), g->stream));
      k_bits_to_queue<<<grid_for(nwords, 256), 256, 0, g->stream>>>(n, front, queue, &c->next_count);
      bottom_up = false;
    }
    GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), g->stream));
    if (!bottom_up) {
      k_frontier_degrees<<<grid_for(nf, 256), 256, 0, g->stream>>>(queue, nf, g->off, deg);
      GRE_CUDA(cub::DeviceScan::ExclusiveSum(cubtmp, cubbytes, deg, prefix, nf + 1, g->stream));
      uint64_t total = 0;
      GRE_CUDA(cudaMemcpyAsync(&total, prefix + nf, sizeof total, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      if (total) {
        int grid = (int)std::min<uint64_t>((total + 255) / 256, (uint64_t)sms * 16);
        k_td_expand<<<grid, 256, 0, g->stream>>>(queue, nf, prefix, total, g->off, g->col, vis, level, d + 1, nqueue, c);
      }
      GRE_LAUNCH_CHECK();
      GRE_CUDA(cudaMemcpyAsync(&h, c, sizeof h, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      h.next_count = h.pad;  // slot counter of warp_append
      scanned_total += total;
      bytes += 16 * nf + 8 * total + 8 * h.next_count;
      std::swap(queue, nqueue);
    } else {
      k_bu_step<<<grid_for(nwords * 32, 256, 8), 256, 0, g->stream>>>(n, g->roff, g->rcol, g->off, front, nbits, vis, level, d + 1, c);
      GRE_LAUNCH_CHECK();
      GRE_CUDA(cudaMemcpyAsync(&h, c, sizeof h, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      scanned_total += h.scanned;
      bytes += 16 * (n - visited) + (uint64_t)(4.125 * (double)h.scanned) + 4 * h.next_count + n / 8;
      std::swap(front, nbits);
    }
    nf = h.next_count;
    mf = h.next_arcs;
    mu -= (int64_t)mf;
    visited += nf;
    ++d;
    if (record) stats_record(st, nf);
  }
  if (st) {
    st->supersteps += (uint32_t)(d > 0 ? d - 1 : 0);  // getSuperstepCount: the empty level is not counted
    st->arcs_traversed += scanned_total;
    st->algo_bytes += bytes;
  }
  return GRE_SUCCESS;
}

// Undirected edges with a reached endpoint: sum over reached v of outdeg(v) / 2 (symmetric).
// sum of the degrees of reached vertices over `rows` level arrays of n entries each
__global__ void k_reached_degree(uint64_t n, uint64_t rows, const int32_t* __restrict__ level, const uint32_t* __restrict__ deg,
                                 unsigned long long* __restrict__ out) {
  unsigned long long s = 0;
  const uint64_t total = n * rows;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x)
    if (level[i] >= 0) s += deg[i % n];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31u) == 0 && s) atomicAdd(out, s);
}

int count_reached_edges(gre_graph g, const int32_t* level, uint64_t* edges, uint64_t rows) {
  unsigned long long* c;
  GRE_CHECK(ws_array(g, WS_COUNTERS, 4, &c));
  GRE_CUDA(cudaMemsetAsync(c, 0, 8, g->stream));
  k_reached_degree<<<grid_for(g->n * rows, 256), 256, 0, g->stream>>>(g->n, rows, level, g->outdeg, c);
  unsigned long long h = 0;
  GRE_CUDA(cudaMemcpyAsync(&h, c, 8, cudaMemcpyDeviceToHost, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  *edges = g->symmetric() ? h / 2 : h;
  return GRE_SUCCESS;
}

// ---------------------------------------------------------------------------------------------
// multi-source BFS, 64 sources per word
// ---------------------------------------------------------------------------------------------
__global__ void k_ms_seed(const uint32_t* __restrict__ srcs, uint32_t k, uint64_t n, unsigned long long* __restrict__ seen,
                          unsigned long long* __restrict__ front, int32_t* __restrict__ levels) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (uint32_t j = 0; j < k; ++j) {
    const uint32_t s = srcs[j];
    seen[s] |= 1ull << j;
    front[s] |= 1ull << j;
    levels[(uint64_t)j * n + s] = 0;
  }
}

// One level: for every vertex with unseen sources, OR the frontier words of its in-neighbours.
// Thread per vertex; stops early once every unseen source has been found.
__global__ void __launch_bounds__(256) k_ms_pull(uint64_t n, uint32_t k, unsigned long long full, const uint64_t* __restrict__ roff,
                                                 const uint32_t* __restrict__ rcol, const unsigned long long* __restrict__ front,
                                                 unsigned long long* __restrict__ next, unsigned long long* __restrict__ seen,
                                                 int32_t* __restrict__ levels, int32_t next_level,
                                                 unsigned long long* __restrict__ counters) {
  unsigned long long found = 0, scanned = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < n; base += stride) {
    const uint64_t v = base + (threadIdx.x & 31u);
    unsigned long long nb = 0;
    if (v < n) {
      const unsigned long long s = seen[v];
      const unsigned long long want = full & ~s;
      if (want) {
        unsigned long long acc = 0;
        const uint64_t a1 = roff[v + 1];
        for (uint64_t a = roff[v]; a < a1; ++a) {
          acc |= front[__ldg(rcol + a)];
          ++scanned;
          if ((acc & want) == want) break;
        }
        nb = acc & want;
      }
      next[v] = nb;
      if (nb) seen[v] = s | nb;
    }
    // levels: all lanes walk the union of their new bits so the writes of one bit coalesce
    unsigned int lo = __reduce_or_sync(0xffffffffu, (unsigned int)(nb & 0xffffffffull));
    unsigned int hi = __reduce_or_sync(0xffffffffu, (unsigned int)(nb >> 32));
    unsigned long long any = ((unsigned long long)hi << 32) | lo;
    while (any) {
      const int j = __ffsll(any) - 1;
      any &= any - 1;
      if ((nb >> j) & 1ull) levels[(uint64_t)j * n + v] = next_level;
    }
    found += __popcll(nb);
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

// Several roots, one search (graphs batched as one block-diagonal union: every root in its own
// component): the roots share source bit 0 of the 64-source word, so the persistent level loop
// of persist.cu runs the whole search in one cooperative launch.  Levels and per-level counts
// equal bfs_levels' (the same levels, found in the same order of levels).  Used on request only
// (see gre_bfs_multiroot).
__global__ void k_ms_seed_roots(const uint32_t* __restrict__ roots, uint32_t k, unsigned long long* __restrict__ seen,
                                unsigned long long* __restrict__ front, int32_t* __restrict__ levels) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
    const uint32_t r = roots[j];
    seen[r] = 1ull;
    front[r] = 1ull;
    levels[r] = 0;
  }
}

static int bfs_multiroot_persistent(gre_graph g, const uint32_t* droots, uint32_t nroots, int32_t* level, gre_stats* st) {
  const uint64_t n = g->n;
  unsigned long long *seen, *fa, *fb, *acc;
  uint32_t *flist, *flist2;
  unsigned char* ctl;
  GRE_CHECK(ws_array(g, WS_A, n, &seen));
  GRE_CHECK(ws_array(g, WS_B, n, &fa));
  GRE_CHECK(ws_array(g, WS_C, n, &fb));
  GRE_CHECK(ws_array(g, WS_E, n, &acc));
  GRE_CHECK(ws_array(g, WS_F, n, &flist));
  GRE_CHECK(ws_array(g, WS_G, n, &flist2));
  GRE_CHECK(ws_array(g, WS_I, msbfs_ctl_bytes(), &ctl));
  GRE_CHECK(ensure_bins(g, true));
  GRE_CUDA(cudaMemsetAsync(level, 0xff, sizeof(int32_t) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(seen, 0, sizeof(unsigned long long) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(fa, 0, sizeof(unsigned long long) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * n, g->stream));
  k_ms_seed_roots<<<grid_for(nroots, 256), 256, 0, g->stream>>>(droots, nroots, seen, fa, level);
  GRE_LAUNCH_CHECK();
  uint32_t nl = 0;
  uint64_t scanned = 0, bytes = 0;
  std::vector<unsigned long long> found;
  GRE_CHECK(msbfs_word_persistent(g, 1ull, seen, fa, fb, acc, flist, flist2, level, ctl,
                                  (unsigned long long*)(ctl + msbfs_ctl_bytes()) - GRE_MAX_RECORDED_SUPERSTEPS, &nl, &scanned,
                                  &bytes, &found));
  for (unsigned long long f : found) stats_record(st, f);
  if (st) {
    st->supersteps += nl;  // the empty level is not counted, as bfs_levels
    st->arcs_traversed += scanned;
    st->algo_bytes += bytes;
  }
  return GRE_SUCCESS;
}

}  // namespace gre

using namespace gre;

extern "C" {

int gre_bfs(gre_graph g, const uint32_t* srcs, uint32_t nsrc, int32_t* levels, gre_stats* st) {
  if (!g || !levels || (nsrc && !srcs)) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  std::vector<uint32_t> hs(nsrc);
  if (nsrc) GRE_CUDA(cudaMemcpy(hs.data(), srcs, sizeof(uint32_t) * nsrc, cudaMemcpyDefault));
  GRE_CHECK(map_ids(g, &hs, "gre_bfs"));
  int32_t *dfinal, *dl;
  uint32_t* droot;
  GRE_CHECK(prepare_output(g, levels, (uint64_t)nsrc * n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, nsrc, 4, (void**)&dl));
  GRE_CHECK(ws_array(g, WS_H, nsrc ? nsrc : 1, &droot));
  RunTimer timer(g);
  if (nsrc) GRE_CUDA(cudaMemcpyAsync(droot, hs.data(), sizeof(uint32_t) * nsrc, cudaMemcpyHostToDevice, g->stream));
  uint64_t edges = 0;
  for (uint32_t i = 0; i < nsrc; ++i) {
    GRE_CHECK(bfs_levels(g, droot + i, 1, dl + (uint64_t)i * n, st, nsrc == 1));
    uint64_t e = 0;
    GRE_CHECK(count_reached_edges(g, dl + (uint64_t)i * n, &e));
    edges += e;
  }
  GRE_CHECK(perm_out_end(g, dl, dfinal, nsrc, 4));
  GRE_CHECK(finish_output(g, levels, dfinal, (uint64_t)nsrc * n));
  GRE_CHECK(timer.stop(st));
  if (st) st->traversed_edges = edges;
  return GRE_SUCCESS;
}

int gre_bfs_multiroot(gre_graph g, const uint32_t* roots, uint32_t nroots, int32_t* level, gre_stats* st) {
  if (!g || !level || (nroots && !roots)) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  std::vector<uint32_t> hs(nroots);
  if (nroots) GRE_CUDA(cudaMemcpy(hs.data(), roots, sizeof(uint32_t) * nroots, cudaMemcpyDefault));
  GRE_CHECK(map_ids(g, &hs, "gre_bfs_multiroot"));
  int32_t *dfinal, *dl;
  uint32_t* droot;
  GRE_CHECK(prepare_output(g, level, n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, 1, 4, (void**)&dl));
  GRE_CHECK(ws_array(g, WS_H, nroots ? nroots : 1, &droot));
  RunTimer timer(g);
  if (nroots) GRE_CUDA(cudaMemcpyAsync(droot, hs.data(), sizeof(uint32_t) * nroots, cudaMemcpyHostToDevice, g->stream));
  // the persistent form only on request (GRE_PERSIST=1): 32 uneven RMAT graphs (scales 12-18,
  // 2.65M vertices, 6 levels) took 1.86 ms against 1.13 ms for the host loop, whose few levels
  // cost less than the persistent loop's 8-byte words per vertex
  const char* pe = getenv("GRE_PERSIST");
  if (nroots > 1 && pe && strtoul(pe, nullptr, 10) != 0 && msbfs_persistent_available(n))
    GRE_CHECK(bfs_multiroot_persistent(g, droot, nroots, dl, st));
  else GRE_CHECK(bfs_levels(g, droot, nroots, dl, st, true));
  uint64_t e = 0;
  GRE_CHECK(count_reached_edges(g, dl, &e));
  GRE_CHECK(perm_out_end(g, dl, dfinal, 1, 4));
  GRE_CHECK(finish_output(g, level, dfinal, n));
  GRE_CHECK(timer.stop(st));
  if (st) st->traversed_edges = e;
  return GRE_SUCCESS;
}

int gre_msbfs(gre_graph g, const uint32_t* srcs, uint32_t nsrc, int32_t* levels, gre_stats* st) {
  if (!g || !levels || (nsrc && !srcs)) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  std::vector<uint32_t> hs(nsrc);
  if (nsrc) GRE_CUDA(cudaMemcpy(hs.data(), srcs, sizeof(uint32_t) * nsrc, cudaMemcpyDefault));
  GRE_CHECK(map_ids(g, &hs, "gre_msbfs"));
  int32_t *dfinal, *dl;
  unsigned long long *seen, *fa, *fb, *cnt;
  uint32_t* dsrc;
  GRE_CHECK(prepare_output(g, levels, (uint64_t)nsrc * n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, nsrc, 4, (void**)&dl));
  GRE_CHECK(ws_array(g, WS_A, n, &seen));
  GRE_CHECK(ws_array(g, WS_B, n, &fa));
  GRE_CHECK(ws_array(g, WS_C, n, &fb));
  unsigned long long* acc;
  uint32_t *flist, *flist2 = nullptr;
  unsigned char* ctl = nullptr;
  GRE_CHECK(ws_array(g, WS_D, 64, &dsrc));
  GRE_CHECK(ws_array(g, WS_E, n, &acc));
  GRE_CHECK(ws_array(g, WS_F, n, &flist));
  GRE_CHECK(ws_array(g, WS_COUNTERS, 8, &cnt));
  GRE_CHECK(ensure_bins(g, true));
  const bool persist = msbfs_persistent_available(n);
  if (persist) {  // the level loop as one cooperative launch per word (persist.cu)
    GRE_CHECK(ws_array(g, WS_G, n, &flist2));
    GRE_CHECK(ws_array(g, WS_H, msbfs_ctl_bytes(), &ctl));
  }
  RunTimer timer(g);
  GRE_CUDA(cudaMemsetAsync(dl, 0xff, sizeof(int32_t) * nsrc * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * n, g->stream));
  uint64_t scanned = 0, bytes = 0;
  uint32_t max_levels = 0;
  for (uint32_t j0 = 0; j0 < nsrc; j0 += 64) {
    const uint32_t k = std::min<uint32_t>(64, nsrc - j0);
    const unsigned long long full = k == 64 ? ~0ull : ((1ull << k) - 1ull);
    GRE_CUDA(cudaMemcpyAsync(dsrc, hs.data() + j0, sizeof(uint32_t) * k, cudaMemcpyHostToDevice, g->stream));
    GRE_CUDA(cudaMemsetAsync(seen, 0, sizeof(unsigned long long) * n, g->stream));
    GRE_CUDA(cudaMemsetAsync(fa, 0, sizeof(unsigned long long) * n, g->stream));
    int32_t* lv = dl + (uint64_t)j0 * n;
    k_ms_seed<<<1, 32, 0, g->stream>>>(dsrc, k, n, seen, fa, lv);
    if (persist) {
      uint32_t nl = 0;
      std::vector<unsigned long long> found;
      GRE_CHECK(msbfs_word_persistent(g, full, seen, fa, fb, acc, flist, flist2, lv, ctl,
                                      (unsigned long long*)(ctl + msbfs_ctl_bytes()) - GRE_MAX_RECORDED_SUPERSTEPS, &nl,
                                      &scanned, &bytes, nsrc <= 64 ? &found : nullptr));
      for (unsigned long long f : found) stats_record(st, f);
      max_levels = std::max<uint32_t>(max_levels, nl);
      continue;
    }
    unsigned long long* front = fa;
    unsigned long long* next = fb;
    unsigned long long live = full;  // sources whose frontier is not empty
    for (int32_t d = 0;; ++d) {
      // direction: push when the frontier's arcs are few (Beamer's rule against all arcs)
      GRE_CUDA(cudaMemsetAsync(cnt, 0, 64, g->stream));
      ms::k_frontier_list<<<grid_for(n, 256, 8), 256, 0, g->stream>>>(n, front, g->off, flist, (unsigned int*)(cnt + 2), cnt + 3);
      unsigned long long h[6];
      GRE_CUDA(cudaMemcpyAsync(h, cnt, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      const bool push = h[3] * 14 < g->m;
      if (push)
        ms::k_push<<<grid_for((h[2] & 0xffffffffull) * 32, 256, 8), 256, 0, g->stream>>>(flist, (unsigned int*)(cnt + 2), g->off,
                                                                                          g->col, front, seen, acc);
      else
        GRE_CHECK(ms::pull(g->bins_in, live, g->roff, g->rcol, front, seen, acc, cnt + 4, g->stream));
      ms::k_commit<<<grid_for(n, 256, 8), 256, 0, g->stream>>>(n, acc, seen, next, lv, d + 1, cnt, cnt + 5);
      GRE_LAUNCH_CHECK();
      GRE_CUDA(cudaMemcpyAsync(h, cnt, sizeof h, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      const unsigned long long found_bits = h[1];
      live = h[5];
      if (push) {
        scanned += h[3];
        bytes += 16 * (h[2] & 0xffffffffull) + 12 * h[3] + 32 * n;
      } else {
        scanned += h[4];
        bytes += 24 * n + 12 * h[4];
      }
      std::swap(front, next);
      if (nsrc <= 64) stats_record(st, found_bits);
      if (found_bits == 0) {
        max_levels = std::max<uint32_t>(max_levels, (uint32_t)d);
        break;
      }
    }
  }
  uint64_t edges = 0;
  GRE_CHECK(count_reached_edges(g, dl, &edges, nsrc));  // all sources in one pass
  GRE_CHECK(perm_out_end(g, dl, dfinal, nsrc, 4));
  GRE_CHECK(finish_output(g, levels, dfinal, (uint64_t)nsrc * n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = max_levels;
    st->arcs_traversed = scanned;
    st->traversed_edges = edges;
    st->algo_bytes = bytes;
  }
  return GRE_SUCCESS;
}

}  // extern "C"
