// 1D-partitioned single-source paths (BFS, PageRank, SSSP, CC): one graph split by vertex over P
// ranks, one GPU each.
//
// The reference at np > 1 gives every vertex one master rank (GraphIngress.hpp:1126-1450) and
// runs a superstep as: sync scatters (masters send their scatter values to the ranks that read
// them, Engine.hpp:273-315), local compute, sync combiners (combined messages return to the
// masters, Engine.hpp:333-374), apply.  Here rank p owns a fixed set of vertex slots together
// with the in-arcs and out-arcs of those vertices (columns global), so a superstep is:
//   * PageRank (pull): scatter-sync = all-gather of the owners' contributions (8 bytes per
//     slot); compute = the degree-binned row reduction of the owned rows (rows.cuh, the same
//     schedule as the whole graph, so every row's sum has the same association order as on one
//     GPU); no combiner-sync.
//   * BFS, bottom-up level: all-gather of the owners' frontier bits (one bit per slot); every
//     owned unvisited vertex looks for a parent among its in-arcs (bfs.cu's k_bu_step on the
//     local rows).
//   * BFS, top-down level: each rank expands its own frontier along out-arcs into a candidate
//     bitmap over all slots; combiner-sync = all-to-all of the bitmap's per-owner blocks; the
//     owner ORs the P blocks it receives and claims the unvisited vertices.
//   * SSSP (near-far): the pending slots below a global limit relax their out-arcs into a
//     candidate array over all slots (sssp.cu's tile kernel, atomic min); combiner-sync =
//     all-to-all of the offers; the owner keeps the smallest and marks improved slots pending.
//   * CC: scatter-sync = all-gather of the labels; every owned row takes the smallest label of
//     its neighbours and of the vertex its label names (label propagation with shortcuts).
// The collectives come from the caller (gre_exchange_fn): the library's own NCCL communicator
// (nccl_exchange.cpp), torch.distributed (graphine_b200/partition.py), or anything else with the
// same all-gather / all-to-all semantics.  Direction rule, levels, distances, labels and
// PageRank values are those of the one-GPU paths.
//
// Vertex layout.  Internal ids are dealt to ranks one by one in snake order: round r = v / P
// gives ranks 0, 1, .., P-1 on even rounds and P-1, .., 1, 0 on odd ones, and vertex v becomes
// slot r of its rank.  On a degree-ordered (relabelled) graph every rank then holds the same
// mix of hubs and leaves, in decreasing degree.  Each rank has L = 64 * ceil(ceil(n / P) / 64)
// slots (whole bitmap words) and the exchange index of slot i of rank p is p * L + i, so every
// per-vertex exchange is a rank-major array of P * L entries built by a plain all-gather of
// equal blocks.  Slots past the last vertex are padding (no arcs, marked visited, never written
// out).
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "gre_internal.cuh"
#include "rows.cuh"
#include "uf.cuh"

struct gre_part_s {
  gre_graph sub = nullptr;   // the owned rows; columns are exchange indices
  uint64_t n = 0, m = 0;     // vertices and arcs of the whole graph
  uint32_t nparts = 1, rank = 0;
  uint64_t L = 0;            // vertex slots per rank (multiple of 64)
  uint64_t arcs_in = 0, arcs_out = 0;  // arcs of the owned rows
  uint32_t* w32 = nullptr;   // weights of the out-arc rows (the graph's, when it had them)
  uint32_t delta = 0;        // SSSP bucket width: the whole graph's (sssp_delta; 0: no buckets)
  uint32_t* xof = nullptr;   // caller id -> exchange index (n)
  uint32_t* xmap = nullptr;  // exchange index -> caller id, 0xffffffff for padding (P * L)
  uint64_t cc_remote = ~0ull;  // arcs of the owned rows that lead to another rank (counted on first use)
  bool w_sym = false;          // the graph's weights are symmetric (w32_symmetric): SSSP may pull
  // SSSP light/heavy split of the owned out-rows for `delta` (built on first use): light arcs first
  uint32_t* sp_col = nullptr;
  uint32_t* sp_w = nullptr;
  uint64_t* sp_lend = nullptr;
};

namespace gre {

struct BfsCounters {
  unsigned long long next_count;
  unsigned long long next_arcs;
  unsigned long long scanned;
  unsigned long long pad;
};

// kernels defined in bfs.cu
__global__ void k_frontier_degrees(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ off,
                                   uint64_t* __restrict__ deg);
__global__ void k_queue_to_bits(const uint32_t* __restrict__ queue, uint64_t nq, uint32_t* __restrict__ bits);
__global__ void __launch_bounds__(256) k_bu_step(uint64_t n, const uint64_t* __restrict__ roff, const uint32_t* __restrict__ rcol,
                                                 const uint64_t* __restrict__ off, const uint32_t* __restrict__ front,
                                                 uint32_t* __restrict__ next, uint32_t* __restrict__ vis, int32_t* __restrict__ level,
                                                 int32_t next_level, BfsCounters* __restrict__ c);
__global__ void k_bits_to_queue(uint64_t n, const uint32_t* __restrict__ bits, uint32_t* __restrict__ queue,
                                unsigned long long* __restrict__ count);

namespace {

template <class T>
int ws_array(gre_graph g, int slot, uint64_t count, T** p) {
  void* v = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &v));
  *p = (T*)v;
  return GRE_SUCCESS;
}

// Exchange index of internal vertex v.
__host__ __device__ __forceinline__ uint64_t part_index(uint64_t v, uint64_t P, uint64_t L) {
  const uint64_t r = v / P, t = v - r * P;
  const uint64_t p = (r & 1) ? P - 1 - t : t;
  return p * L + r;
}

// Internal vertex of slot i of rank p (>= n: padding).
__host__ __device__ __forceinline__ uint64_t part_vertex(uint64_t i, uint64_t p, uint64_t P) {
  return i * P + ((i & 1) ? P - 1 - p : p);
}

__host__ __device__ __forceinline__ uint64_t part_slots(uint64_t n, uint64_t P) {
  const uint64_t per = (n + P - 1) / P;
  return 64 * (per ? (per + 63) / 64 : 1);
}

__global__ void k_part_maps(uint64_t n, uint64_t P, uint64_t L, const uint32_t* __restrict__ perm, uint32_t* __restrict__ xof,
                            uint32_t* __restrict__ xmap) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = perm ? perm[v] : (uint32_t)v;
    const uint32_t x = (uint32_t)part_index(v, P, L);
    xof[c] = x;
    xmap[x] = c;
  }
}

// deg[i] = arcs of slot i (L + 1 entries, the last 0, for the exclusive scan); deg32 optional
__global__ void k_part_degrees(uint64_t L, uint64_t p, uint64_t P, uint64_t n, const uint64_t* __restrict__ off,
                               uint64_t* __restrict__ deg, uint32_t* __restrict__ deg32) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= L; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t v = i < L ? part_vertex(i, p, P) : n;
    const uint64_t d = v < n ? off[v + 1] - off[v] : 0;
    deg[i] = d;
    if (deg32 && i < L) deg32[i] = (uint32_t)d;
  }
}

// Arcs of every slot copied in stored order, columns turned into exchange indices; warp per row.
__global__ void __launch_bounds__(256) k_part_rows(uint64_t L, uint64_t p, uint64_t P, uint64_t n, const uint64_t* __restrict__ off,
                                                   const uint32_t* __restrict__ col, const uint64_t* __restrict__ loff,
                                                   uint32_t* __restrict__ lcol) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t i = warp; i < L; i += nwarps) {
    const uint64_t v = part_vertex(i, p, P);
    if (v >= n) continue;
    const uint64_t a0 = off[v], len = off[v + 1] - a0, dst = loff[i];
    for (uint64_t k = lane; k < len; k += 32) lcol[dst + k] = (uint32_t)part_index(__ldg(col + a0 + k), P, L);
  }
}

// padding slots (internal id >= n) start visited
__global__ void k_part_pad_visited(uint64_t L, uint64_t p, uint64_t P, uint64_t n, uint32_t* __restrict__ vis) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x)
    if (part_vertex(i, p, P) >= n) atomicOr(vis + (i >> 5), 1u << (i & 31u));
}

__global__ void k_part_seed(uint64_t slot, int32_t* __restrict__ level, uint32_t* __restrict__ vis, uint32_t* __restrict__ queue,
                            const uint32_t* __restrict__ outdeg, BfsCounters* __restrict__ c) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  level[slot] = 0;
  vis[slot >> 5] |= 1u << (slot & 31u);
  queue[0] = (uint32_t)slot;
  c->next_count = 1;
  c->next_arcs = outdeg[slot];
}

// Top-down: one thread per arc of the local frontier (prefix = exclusive scan of its degrees);
// the target's bit is set in the candidate bitmap over all P * L slots.
__global__ void __launch_bounds__(256) k_part_expand(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ prefix,
                                                     uint64_t total, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                     uint32_t* __restrict__ cand) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = nq;
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) >> 1;
      if (prefix[mid] <= t) lo = mid;
      else hi = mid;
    }
    const uint32_t u = queue[lo];
    const uint32_t x = __ldg(col + off[u] + (t - prefix[lo]));
    const uint32_t bit = 1u << (x & 31u);
    if (!(cand[x >> 5] & bit)) atomicOr(cand + (x >> 5), bit);
  }
}

// Top-down claim on the owner: OR of the P received blocks (W words each), minus the visited
// bits; claimed slots get the level and go to the next queue (in slot order within a warp).
__global__ void k_part_claim(uint64_t W, uint64_t P, const uint32_t* __restrict__ recv, uint32_t* __restrict__ vis,
                             int32_t* __restrict__ level, int32_t next_level, const uint32_t* __restrict__ outdeg,
                             uint32_t* __restrict__ queue, BfsCounters* __restrict__ c) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long arcs = 0;
  for (uint64_t base = tid - lane; base < W; base += nthreads) {
    const uint64_t w = base + lane;
    uint32_t word = 0;
    if (w < W) {
      for (uint64_t q = 0; q < P; ++q) word |= recv[q * W + w];
      const uint32_t old = vis[w];
      word &= ~old;
      if (word) vis[w] = old | word;
    }
    const uint32_t cnt = __popc(word);
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long pos = 0;
    if (lane == 31 && total) pos = atomicAdd(&c->next_count, (unsigned long long)total);
    pos = __shfl_sync(0xffffffffu, pos, 31) + incl - cnt;
    uint32_t x = word;
    while (x) {
      const uint32_t b = __ffs(x) - 1;
      x &= x - 1;
      const uint32_t i = (uint32_t)(w << 5) + b;
      level[i] = next_level;
      arcs += outdeg[i];
      queue[pos++] = i;
    }
  }
  for (int o = 16; o > 0; o >>= 1) arcs += __shfl_xor_sync(0xffffffffu, arcs, o);
  if (lane == 0 && arcs) atomicAdd(&c->next_arcs, arcs);
}

// sum of the out-degrees of reached slots (edges with a reached endpoint)
__global__ void k_part_reached(uint64_t L, const int32_t* __restrict__ level, const uint32_t* __restrict__ deg,
                               unsigned long long* __restrict__ out) {
  unsigned long long s = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x)
    if (level[i] >= 0) s += deg[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31u) == 0 && s) atomicAdd(out, s);
}

// sum of the out-degrees of slots with a finite distance
__global__ void k_part_reached_dist(uint64_t L, const uint32_t* __restrict__ dist, const uint32_t* __restrict__ deg,
                                    unsigned long long* __restrict__ out) {
  unsigned long long s = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x)
    if (dist[i] != 0xffffffffu) s += deg[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31u) == 0 && s) atomicAdd(out, s);
}

// gathered rank-major values -> caller order
template <class T>
__global__ void k_part_out(uint64_t total, const uint32_t* __restrict__ xmap, const T* __restrict__ in, T* __restrict__ out) {
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total; x += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = xmap[x];
    if (c != 0xffffffffu) out[c] = in[x];
  }
}

struct PartGather {
  const uint32_t* __restrict__ col;
  const double* __restrict__ contrib;  // all P * L slots
  __device__ __forceinline__ double operator()(uint32_t, uint64_t a) const { return __ldg(contrib + __ldg(col + a)); }
};

// pr = tele + d * sum; the power iteration refreshes the owner's contribution pr / outdeg
struct PartFinish {
  double* __restrict__ pr;
  double* __restrict__ contrib;  // null: never refreshed (reference variant)
  const uint32_t* __restrict__ outdeg;
  double tele, d;
  __device__ __forceinline__ void operator()(uint32_t v, double sum) const {
    const double x = tele + d * sum;
    pr[v] = x;
    if (contrib) {
      const uint32_t od = outdeg[v];
      contrib[v] = od ? x / (double)od : 0.0;
    }
  }
};

__global__ void k_part_pr_init(uint64_t L, const uint32_t* __restrict__ outdeg, double tele, double* __restrict__ pr,
                               double* __restrict__ contrib) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t od = outdeg[i];
    pr[i] = tele;
    contrib[i] = od ? tele / (double)od : 0.0;
  }
}

// Arc weights of the slots' rows in stored order (the same order as k_part_rows).
__global__ void __launch_bounds__(256) k_part_weights(uint64_t L, uint64_t p, uint64_t P, uint64_t n,
                                                      const uint64_t* __restrict__ off, const uint32_t* __restrict__ w,
                                                      const uint64_t* __restrict__ loff, uint32_t* __restrict__ lw) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t i = warp; i < L; i += nwarps) {
    const uint64_t v = part_vertex(i, p, P);
    if (v >= n) continue;
    const uint64_t a0 = off[v], len = off[v + 1] - a0, dst = loff[i];
    for (uint64_t k = lane; k < len; k += 32) lw[dst + k] = __ldg(w + a0 + k);
  }
}

// SSSP claim on the owner: the smallest of the P offers for each slot; an improvement lowers the
// distance and marks the slot pending (to be relaxed when its bucket comes; slots without
// out-arcs never are).  One warp covers 32 consecutive slots, i.e. one pending word.
__global__ void k_part_sssp_claim(uint64_t L, uint64_t P, const uint32_t* __restrict__ recv, uint32_t* __restrict__ dist,
                                  const uint32_t* __restrict__ outdeg, uint32_t* __restrict__ pend) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < L; base += stride) {
    const uint64_t i = base + (threadIdx.x & 31u);
    bool mark = false;
    if (i < L) {
      uint32_t m = 0xffffffffu;
      for (uint64_t q = 0; q < P; ++q) m = min(m, recv[q * L + i]);
      if (m < dist[i]) {
        dist[i] = m;
        mark = outdeg[i] != 0;
      }
    }
    const uint32_t ball = __ballot_sync(0xffffffffu, mark);
    if ((threadIdx.x & 31u) == 0 && ball) pend[base >> 5] |= ball;
  }
}

// Near-far selection with the light/heavy split of delta-stepping (Davidson et al., IPDPS 2014;
// Meyer and Sanders 2003), as the one-GPU path.  The slots improved since the last selection
// (bits of `pend`, cleared here) and, right after the limit rose, every slot of the far set
// (bitmap `farb`) are examined: below the limit a slot leaves the far set; with light arcs
// ([off, lend)) it joins this superstep's light frontier, with heavy arcs ([lend, off+1)) the
// bucket, whose heavy arcs are relaxed once when no rank has a light frontier left.  At or above
// the limit it joins (or stays in) the far set.  `pending` counts the far set; `min_far` is the
// smallest distance seen going far (exact after a rescan, a lower bound otherwise: the host
// passes the previous value in).  One lane owns each word.
struct SsspCounters {
  unsigned long long near;        // light frontier of this superstep
  unsigned long long pending;     // slots of the far set (at or above the limit)
  unsigned long long min_far;     // smallest far distance (see above)
  unsigned long long arcs;        // light arcs of the frontier
  unsigned long long bucket_new;  // slots that joined the bucket
  unsigned long long heavy_new;   // their heavy arcs
  unsigned long long pad[2];
};

__global__ void __launch_bounds__(256) k_part_sssp_select(uint64_t W, uint32_t* __restrict__ pend, uint32_t* __restrict__ farb,
                                                          bool rescan, const uint32_t* __restrict__ dist, uint32_t limit,
                                                          const uint64_t* __restrict__ off, const uint64_t* __restrict__ lend,
                                                          uint32_t* __restrict__ inb, uint32_t* __restrict__ queue,
                                                          SsspCounters* __restrict__ c) {
  __shared__ uint32_t stage[8][1024];
  WarpLists<1, 1024> out(stage[threadIdx.x >> 5]);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long left = 0, arcs = 0, joined = 0, heavy = 0;
  uint32_t dmin = 0xffffffffu;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < W; base += stride) {
    const uint64_t w = base + (threadIdx.x & 31u);
    const uint32_t nb = w < W ? pend[w] : 0u, fb = w < W ? farb[w] : 0u;
    uint32_t bits = rescan ? nb | fb : nb, far_now = fb, join = 0;
    const uint32_t inw = bits ? inb[w] : 0u;
    while (__any_sync(0xffffffffu, bits != 0)) {
      bool take = false;
      uint32_t i = 0;
      if (bits) {
        const uint32_t b = __ffs(bits) - 1;
        bits &= bits - 1;
        i = (uint32_t)(w << 5) + b;
        const uint32_t d = dist[i];
        if (d < limit) {
          far_now &= ~(1u << b);
          const uint64_t a0 = off[i], am = lend[i], a1 = off[i + 1];
          take = am > a0;
          arcs += am - a0;
          if (a1 > am && !((inw >> b) & 1u)) {
            join |= 1u << b;
            heavy += a1 - am;
          }
        } else {
          far_now |= 1u << b;
          dmin = min(dmin, d);
        }
      }
      out.push<0>(take, i, (uint32_t*)&c->near, queue);
    }
    if (nb) pend[w] = 0;
    if (far_now != fb) farb[w] = far_now;
    left += __popc(far_now);
    if (join) {
      inb[w] = inw | join;
      joined += __popc(join);
    }
  }
  out.flush<0>((uint32_t*)&c->near, queue);
  dmin = __reduce_min_sync(0xffffffffu, dmin);
  for (int o = 16; o > 0; o >>= 1) {
    left += __shfl_xor_sync(0xffffffffu, left, o);
    arcs += __shfl_xor_sync(0xffffffffu, arcs, o);
    joined += __shfl_xor_sync(0xffffffffu, joined, o);
    heavy += __shfl_xor_sync(0xffffffffu, heavy, o);
  }
  if ((threadIdx.x & 31u) == 0) {
    if (left) atomicAdd(&c->pending, left);
    if (arcs) atomicAdd(&c->arcs, arcs);
    if (joined) atomicAdd(&c->bucket_new, joined);
    if (heavy) atomicAdd(&c->heavy_new, heavy);
    if (dmin != 0xffffffffu) atomicMin(&c->min_far, (unsigned long long)dmin);
  }
}

// Offer slots written since the last clear (bits in `touched`, one per slot of all P * L) go back
// to "no offer", and the bits are cleared: the offer array is reset without a full memset.
__global__ void k_part_offers_clear(uint64_t words, uint32_t* __restrict__ touched, uint32_t* __restrict__ cand) {
  for (uint64_t wi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; wi < words; wi += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t bits = touched[wi];
    if (!bits) continue;
    touched[wi] = 0;
    while (bits) {
      const uint32_t b = __ffs(bits) - 1;
      bits &= bits - 1;
      cand[(wi << 5) + b] = 0xffffffffu;
    }
  }
}

// The offers of one superstep as per-owner lists, for a superstep whose offers are few: owner q's
// block (`block` uint2 from send + q * block) holds its count in .x of the first element, then
// (slot within q's part, distance) pairs of the offer slots written since the last clear.  The
// slots go back to "no offer" and their bits are cleared, as k_part_offers_clear.  The offers of
// a superstep are at most its arcs, the bound the host sizes `cap` by; a pair past `cap` would
// set *err and be dropped.  grid.y = owner; a warp appends its 32 words' pairs with one atomic.
__global__ void k_part_offers_pack(uint64_t W, uint32_t* __restrict__ touched, uint32_t* __restrict__ cand,
                                   uint2* __restrict__ send, uint64_t block, uint64_t cap, uint32_t* __restrict__ err) {
  const uint64_t q = blockIdx.y;
  uint32_t* tq = touched + q * W;
  uint32_t* cq = cand + q * W * 32;
  uint2* out = send + q * block;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < W; base += stride) {
    const uint64_t wi = base + lane;
    uint32_t bits = wi < W ? tq[wi] : 0u;
    if (!__any_sync(0xffffffffu, bits != 0)) continue;
    const uint32_t k = __popc(bits);
    uint32_t incl = k;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t at = 0;
    if (lane == 0) at = atomicAdd(&out[0].x, total);
    at = __shfl_sync(0xffffffffu, at, 0) + incl - k;
    if (bits) tq[wi] = 0;
    while (bits) {
      const uint32_t b = __ffs(bits) - 1;
      bits &= bits - 1;
      const uint32_t slot = (uint32_t)(wi << 5) + b;
      if (at < cap) {
        out[1 + at] = make_uint2(slot, cq[slot]);
      } else {
        atomicOr(err, 2u);
      }
      cq[slot] = 0xffffffffu;
      ++at;
    }
  }
}

// SSSP claim from per-owner lists (k_part_offers_pack's blocks, one from each rank): the distance
// of each offered slot becomes the smallest of its offers and an improved slot with out-arcs is
// marked pending, as k_part_sssp_claim does from the dense offer arrays.  A count above `cap` or
// a slot past L (never written by the pack) sets *err and is not read.
__global__ void k_part_sssp_claim_lists(uint64_t P, uint64_t L, const uint2* __restrict__ recv, uint64_t block, uint64_t cap,
                                        uint32_t* __restrict__ dist, const uint32_t* __restrict__ outdeg,
                                        uint32_t* __restrict__ pend, uint32_t* __restrict__ err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = 0; q < P; ++q) {
    const uint2* in = recv + q * block;
    uint64_t cnt = in[0].x;
    if (cnt > cap) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, 2u);
      cnt = cap;
    }
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += stride) {
      const uint2 o = in[1 + i];
      if (o.x >= L) {
        atomicOr(err, 2u);
        continue;
      }
      if (o.y < atomicMin(dist + o.x, o.y) && outdeg[o.x]) atomicOr(pend + (o.x >> 5), 1u << (o.x & 31u));
    }
  }
}

// arcs of the queued slots in their light ([off, lend)) or heavy ([lend, off+1)) range
__global__ void k_part_range_degrees(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ off,
                                     const uint64_t* __restrict__ lend, bool heavy, uint64_t* __restrict__ deg) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = queue[i];
    deg[i] = heavy ? off[v + 1] - lend[v] : lend[v] - off[v];
  }
}

// CC, phase 1: union-find over the arcs whose both ends this rank owns (slots lo .. lo + L - 1
// in exchange indices), roots linked by the caller id of the slot (key).
struct HookLocal {
  const uint32_t* __restrict__ col;  // exchange indices
  uint32_t* parent;                  // L slots
  const uint32_t* __restrict__ key;  // caller id of each slot
  uint32_t lo, L;
  // Afforest's second pass (symmetric graphs): rows flagged in `skip` are left out and the first
  // `sampled` arcs of the others were already seen (null: every arc)
  const uint32_t* __restrict__ skip = nullptr;
  const uint64_t* __restrict__ off = nullptr;
  uint32_t sampled = 0;
  __device__ __forceinline__ double operator()(uint32_t u, uint64_t a) const {
    if (skip) {
      if ((__ldg(skip + (u >> 5)) >> (u & 31u)) & 1u) return 0.0;
      if (a < __ldg(off + u) + sampled) return 0.0;
    }
    const uint32_t x = __ldg(col + a) - lo;  // wraps past L for remote slots
    if (x < L) uf_union(parent, key, u, x);
    return 0.0;
  }
};

struct NoFinishPart {
  __device__ __forceinline__ void operator()(uint32_t, double) const {}
};

// Afforest's first pass over the local arcs: every slot united with the local ones among its
// first k arcs (the hubs, on a relabelled graph)
__global__ void k_pcc_sample(uint64_t L, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col, uint32_t k,
                             uint32_t lo, uint32_t* parent, const uint32_t* __restrict__ key) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < L; u += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a0 = off[u], a1 = off[u + 1];
    for (uint64_t a = a0; a < a1 && a < a0 + k; ++a) {
      const uint32_t x = __ldg(col + a) - lo;
      if (x < L) uf_union(parent, key, (uint32_t)u, x);
    }
  }
}

// arcs of the rows that lead to another rank's slots
__global__ void k_pcc_count_remote(uint64_t arcs, const uint32_t* __restrict__ col, uint32_t lo, uint32_t L,
                                   unsigned long long* __restrict__ out) {
  unsigned long long c = 0;
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < arcs; a += (uint64_t)gridDim.x * blockDim.x)
    c += (uint32_t)(__ldg(col + a) - lo) >= L;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31u) == 0 && c) atomicAdd(out, c);
}

// after phase 1 (parent[i] = root of i): every slot's label is its root's key, every root's
// component label too
__global__ void k_pcc_labels(uint64_t L, const uint32_t* __restrict__ parent, const uint32_t* __restrict__ key,
                             uint32_t* __restrict__ lab, uint32_t* __restrict__ rootlab) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = parent[i];
    lab[i] = key[r];
    if (r == i) rootlab[i] = key[i];
  }
}

// CC, phase 2 (one round): the smallest label behind the row's remote arcs (labels of all slots
// from the round's all-gather) offered to the row's local component.  G lanes per row.
template <int G>
__global__ void __launch_bounds__(256) k_pcc_cut_lanes(const uint32_t* __restrict__ rows, uint64_t count,
                                                       const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                       uint32_t lo, uint32_t L, const uint32_t* __restrict__ lab_all,
                                                       const uint32_t* __restrict__ parent, uint32_t* __restrict__ rootlab) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint32_t lig = threadIdx.x % G;
  const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x) / G;
  // warp-uniform trip count: every lane takes part in the shuffles
  for (uint64_t base = (tid / G) & ~(uint64_t)(32 / G - 1); base < count; base += ngroups) {
    const uint64_t r = base + (threadIdx.x & 31u) / G;
    uint32_t m = 0xffffffffu, v = 0;
    if (r < count) {
      v = rows[r];
      for (uint64_t a = off[v] + lig; a < off[v + 1]; a += G) {
        const uint32_t x = __ldg(col + a);
        if (x - lo >= L) m = min(m, lab_all[x]);
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (r < count && lig == 0 && m != 0xffffffffu) {
      const uint32_t root = parent[v];
      if (m < rootlab[root]) atomicMin(rootlab + root, m);
    }
  }
}

// the same for the long rows (bins 6-7): CTA per row
__global__ void __launch_bounds__(256) k_pcc_cut_rows(const uint32_t* __restrict__ rows, uint64_t count,
                                                      const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                      uint32_t lo, uint32_t L, const uint32_t* __restrict__ lab_all,
                                                      const uint32_t* __restrict__ parent, uint32_t* __restrict__ rootlab) {
  for (uint64_t r = blockIdx.x; r < count; r += gridDim.x) {
    const uint32_t v = rows[r];
    uint32_t m = 0xffffffffu;
    for (uint64_t a = off[v] + threadIdx.x; a < off[v + 1]; a += blockDim.x) {
      const uint32_t x = __ldg(col + a);
      if (x - lo >= L) m = min(m, lab_all[x]);
    }
    m = __reduce_min_sync(0xffffffffu, m);
    if ((threadIdx.x & 31u) == 0 && m != 0xffffffffu) {
      const uint32_t root = parent[v];
      if (m < rootlab[root]) atomicMin(rootlab + root, m);
    }
  }
}

// roots: the shortcut through the vertex the label names (its label in the round's snapshot)
__global__ void k_pcc_roots(uint64_t L, const uint32_t* __restrict__ parent, const uint32_t* __restrict__ lab_all,
                            const uint32_t* __restrict__ xof, uint32_t* __restrict__ rootlab) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x) {
    if (parent[i] != i) continue;
    const uint32_t l = rootlab[i];
    if (l == 0xffffffffu) continue;  // padding
    const uint32_t s = lab_all[xof[l]];
    if (s < l) rootlab[i] = s;
  }
}

// members take their component's label; c->next_count += slots whose label dropped
__global__ void k_pcc_members(uint64_t L, const uint32_t* __restrict__ parent, const uint32_t* __restrict__ rootlab,
                              uint32_t* __restrict__ lab, BfsCounters* __restrict__ c) {
  unsigned long long changed = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < L; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t l = rootlab[parent[i]];
    if (l < lab[i]) {
      lab[i] = l;
      ++changed;
    }
  }
  for (int o = 16; o > 0; o >>= 1) changed += __shfl_xor_sync(0xffffffffu, changed, o);
  if ((threadIdx.x & 31u) == 0 && changed) atomicAdd(&c->next_count, changed);
}

// Rows of slots [0, L) of rank p from (off, col): *loff (L + 1) and *lcol allocated here.
int part_rows(gre_graph s, uint64_t p, uint64_t P, uint64_t n, const uint64_t* off, const uint32_t* col, uint64_t** loff,
              uint32_t** lcol, uint32_t** deg32, uint64_t* arcs) {
  const uint64_t L = s->n;
  uint64_t* deg = nullptr;
  GRE_CHECK(ws_array(s, WS_A, L + 1, &deg));
  GRE_CUDA(cudaMalloc(loff, sizeof(uint64_t) * (L + 1)));
  GRE_CUDA(cudaMalloc(deg32, sizeof(uint32_t) * L));
  k_part_degrees<<<grid_for(L + 1, 256), 256, 0, s->stream>>>(L, p, P, n, off, deg, *deg32);
  size_t tb = 0;
  void* tmp = nullptr;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, deg, *loff, L + 1, s->stream);
  GRE_CHECK(s->ws.get(WS_CUB, tb, &tmp));
  GRE_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, deg, *loff, L + 1, s->stream));
  GRE_CUDA(cudaMemcpyAsync(arcs, *loff + L, sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream));
  GRE_CUDA(cudaStreamSynchronize(s->stream));
  GRE_CUDA(cudaMalloc(lcol, sizeof(uint32_t) * (*arcs ? *arcs : 1)));
  k_part_rows<<<grid_for(L * 32, 256, 8), 256, 0, s->stream>>>(L, p, P, n, off, col, *loff, *lcol);
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

// One collective through the caller's exchange; a failure there becomes GRE_FAILURE.
int exchange(gre_part p, gre_exchange_fn xchg, void* ctx, int kind, const void* send, void* recv, uint64_t bytes) {
  const int r = xchg(ctx, kind, send, recv, bytes, (void*)p->sub->stream);
  if (r) {
    set_error("gre_part: the exchange callback returned %d (kind %d, %llu bytes per rank)", r, kind, (unsigned long long)bytes);
    return GRE_FAILURE;
  }
  return GRE_SUCCESS;
}

// Counters of all ranks: local values in, sums (and this rank's entry) out.
int exchange_counters(gre_part p, gre_exchange_fn xchg, void* ctx, BfsCounters* c, BfsCounters* all, BfsCounters* sum,
                      BfsCounters* mine) {
  GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, c, all, sizeof(BfsCounters)));
  std::vector<BfsCounters> h(p->nparts);
  GRE_CUDA(cudaMemcpyAsync(h.data(), all, sizeof(BfsCounters) * p->nparts, cudaMemcpyDeviceToHost, p->sub->stream));
  GRE_CUDA(cudaStreamSynchronize(p->sub->stream));
  *sum = BfsCounters{0, 0, 0, 0};
  for (const BfsCounters& x : h) {
    sum->next_count += x.next_count;
    sum->next_arcs += x.next_arcs;
    sum->scanned += x.scanned;
  }
  if (mine) *mine = h[p->rank];
  return GRE_SUCCESS;
}

void destroy_part(gre_part p) {
  if (!p) return;
  if (p->sub) {
    cudaSetDevice(p->sub->device);
    cudaFree(p->xof);
    cudaFree(p->xmap);
    cudaFree(p->w32);
    cudaFree(p->sp_col);
    cudaFree(p->sp_w);
    cudaFree(p->sp_lend);
    destroy_graph(p->sub);
  }
  delete p;
}

}  // namespace
}  // namespace gre

using namespace gre;

extern "C" {

int gre_part_create(gre_graph g, uint32_t nparts, uint32_t rank, gre_part* out) {
  if (!g || !out) return GRE_NULL;
  *out = nullptr;
  if (nparts == 0 || rank >= nparts) {
    set_error("gre_part_create: rank %u of %u parts", rank, nparts);
    return GRE_INVALID_ARG;
  }
  GRE_CHECK(use_graph(g));
  GRE_CUDA(cudaStreamSynchronize(g->stream));  // the part's stream reads g's arrays
  const uint64_t n = g->n, P = nparts;
  const uint64_t L = part_slots(n, P);
  if (P * L > 0xffffffffull) {
    set_error("gre_part_create: %llu slots exceed 32-bit vertex ids", (unsigned long long)(P * L));
    return GRE_INVALID_ARG;
  }
  // the whole graph's schedule, without source windows (those split rows by column)
  GRE_CHECK(ensure_bins(g, true));
  RowSchedule sched = g->bins_in.sched;
  sched.seg_window = 0;
  gre_part p = new gre_part_s;
  p->n = n;
  p->m = g->m;
  p->nparts = nparts;
  p->rank = rank;
  p->L = L;
  int st = new_graph(g->device, g->flags & ~(uint32_t)GRE_GRAPH_REORDER, &p->sub);
  if (st) {
    delete p;
    return st;
  }
  auto build = [&]() -> int {
    gre_graph s = p->sub;
    s->n = L;
    GRE_CHECK(part_rows(s, rank, P, n, g->roff, g->rcol, &s->roff, &s->rcol, &s->indeg, &p->arcs_in));
    if (g->symmetric()) {
      s->off = s->roff;
      s->col = s->rcol;
      s->outdeg = s->indeg;
      p->arcs_out = p->arcs_in;
    } else {
      GRE_CHECK(part_rows(s, rank, P, n, g->off, g->col, &s->off, &s->col, &s->outdeg, &p->arcs_out));
    }
    s->m = p->arcs_out;
    if (g->w32) {
      GRE_CUDA(cudaMalloc(&p->w32, sizeof(uint32_t) * (p->arcs_out ? p->arcs_out : 1)));
      k_part_weights<<<grid_for(L * 32, 256, 8), 256, 0, s->stream>>>(L, rank, P, n, g->off, g->w32, s->off, p->w32);
      GRE_LAUNCH_CHECK();
      GRE_CHECK(sssp_delta(g, &p->delta));  // the whole graph's, the same on every rank
      p->w_sym = g->w32_symmetric && g->symmetric();
    }
    GRE_CUDA(cudaMalloc(&p->xof, sizeof(uint32_t) * (n ? n : 1)));
    GRE_CUDA(cudaMalloc(&p->xmap, sizeof(uint32_t) * P * L));
    GRE_CUDA(cudaMemsetAsync(p->xmap, 0xff, sizeof(uint32_t) * P * L, s->stream));
    if (n) k_part_maps<<<grid_for(n, 256), 256, 0, s->stream>>>(n, P, L, g->perm, p->xof, p->xmap);
    GRE_LAUNCH_CHECK();
    // the row kernels read the CSC rows (build_bins works on s->n = L rows)
    GRE_CHECK(build_bins(s, s->bins_in, s->roff, s->rcol, sched));
    if (!g->symmetric()) GRE_CHECK(build_bins(s, s->bins_out, s->off, s->col, sched));  // CC pulls both ways
    GRE_CUDA(cudaStreamSynchronize(s->stream));
    return GRE_SUCCESS;
  };
  st = build();
  if (st) {
    destroy_part(p);
    return st;
  }
  *out = p;
  return GRE_SUCCESS;
}

int gre_part_layout(uint64_t n, uint32_t nparts, uint64_t* slots, uint32_t* index) {
  if (!slots) return GRE_NULL;
  if (nparts == 0) return GRE_INVALID_ARG;
  const uint64_t P = nparts, L = part_slots(n, P);
  if (P * L > 0xffffffffull) return GRE_INVALID_ARG;
  *slots = L;
  if (index)
    for (uint64_t v = 0; v < n; ++v) index[v] = (uint32_t)part_index(v, P, L);
  return GRE_SUCCESS;
}

int gre_part_free(gre_part p) {
  destroy_part(p);
  return GRE_SUCCESS;
}

int gre_part_info(gre_part p, uint64_t* slots, uint64_t* arcs_in, uint64_t* arcs_out) {
  if (!p) return GRE_NULL;
  if (slots) *slots = p->L;
  if (arcs_in) *arcs_in = p->arcs_in;
  if (arcs_out) *arcs_out = p->arcs_out;
  return GRE_SUCCESS;
}

int gre_part_bfs(gre_part p, uint32_t src, int32_t* level, gre_exchange_fn xchg, void* ctx, gre_stats* st) {
  if (!p || !level || !xchg) return GRE_NULL;
  gre_graph s = p->sub;
  GRE_CHECK(use_graph(s));
  stats_reset(st);
  const uint64_t n = p->n, P = p->nparts, L = p->L, W = L / 32, me = p->rank;
  if (src >= n) {
    set_error("gre_part_bfs: source %u out of range (n = %llu)", src, (unsigned long long)n);
    return GRE_INVALID_ARG;
  }
  int32_t *lvl, *lvl_all, *dout;
  uint32_t *vis, *queue, *nqueue, *front, *next, *front_all, *cand, *recv;
  uint64_t *deg, *prefix;
  BfsCounters *c, *call;
  GRE_CHECK(ws_array(s, WS_A, L, &lvl));
  GRE_CHECK(ws_array(s, WS_B, P * L, &lvl_all));
  GRE_CHECK(ws_array(s, WS_C, W, &vis));
  GRE_CHECK(ws_array(s, WS_D, L, &queue));
  GRE_CHECK(ws_array(s, WS_E, L, &nqueue));
  GRE_CHECK(ws_array(s, WS_F, W, &front));
  GRE_CHECK(ws_array(s, WS_G, W, &next));
  GRE_CHECK(ws_array(s, WS_H, P * W, &front_all));
  GRE_CHECK(ws_array(s, WS_I, P * W, &cand));
  GRE_CHECK(ws_array(s, WS_J, P * W, &recv));
  GRE_CHECK(ws_array(s, WS_K, L + 1, &deg));
  GRE_CHECK(ws_array(s, WS_L, L + 1, &prefix));
  GRE_CHECK(ws_array(s, WS_COUNTERS, 1, &c));
  GRE_CHECK(ws_array(s, WS_OUTBUF2, P, &call));
  GRE_CHECK(prepare_output(s, level, n, WS_OUTBUF, &dout));
  void* cubtmp = nullptr;
  size_t cubbytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cubbytes, deg, prefix, L + 1, s->stream);
  GRE_CHECK(s->ws.get(WS_CUB, cubbytes, &cubtmp));

  RunTimer timer(s);
  uint32_t xr = 0;
  GRE_CUDA(cudaMemcpyAsync(&xr, p->xof + src, sizeof xr, cudaMemcpyDeviceToHost, s->stream));
  GRE_CUDA(cudaMemsetAsync(lvl, 0xff, sizeof(int32_t) * L, s->stream));
  GRE_CUDA(cudaMemsetAsync(vis, 0, sizeof(uint32_t) * W, s->stream));
  GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), s->stream));
  k_part_pad_visited<<<grid_for(L, 256), 256, 0, s->stream>>>(L, me, P, n, vis);
  GRE_CUDA(cudaStreamSynchronize(s->stream));
  uint64_t nq = 0;  // local queue length
  if (xr / L == me) {
    k_part_seed<<<1, 32, 0, s->stream>>>(xr - me * L, lvl, vis, queue, s->outdeg, c);
    nq = 1;
  }
  GRE_LAUNCH_CHECK();
  BfsCounters sum, mine;
  GRE_CHECK(exchange_counters(p, xchg, ctx, c, call, &sum, &mine));
  uint64_t nf = sum.next_count, mf = sum.next_arcs;
  int64_t mu = (int64_t)p->m - (int64_t)mf;
  bool bottom_up = false;
  int32_t d = 0;
  uint64_t scanned_total = 0, bytes = 0, visited = nf;
  const int sms = num_sms();
  while (nf > 0) {
    // direction choice on global counts: every rank takes the same branch
    if (!bottom_up && (double)mf > (double)mu / 15.0 && nf > 64) {
      GRE_CUDA(cudaMemsetAsync(front, 0, sizeof(uint32_t) * W, s->stream));
      if (nq) k_queue_to_bits<<<grid_for(nq, 256), 256, 0, s->stream>>>(queue, nq, front);
      GRE_LAUNCH_CHECK();
      GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, front, front_all, 4 * W));
      bottom_up = true;
    } else if (bottom_up && nf < n / 18) {
      GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), s->stream));
      k_bits_to_queue<<<grid_for(W, 256), 256, 0, s->stream>>>(L, front, queue, &c->next_count);
      GRE_LAUNCH_CHECK();
      unsigned long long h = 0;
      GRE_CUDA(cudaMemcpyAsync(&h, &c->next_count, sizeof h, cudaMemcpyDeviceToHost, s->stream));
      GRE_CUDA(cudaStreamSynchronize(s->stream));
      nq = h;
      bottom_up = false;
    }
    GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), s->stream));
    if (!bottom_up) {
      GRE_CUDA(cudaMemsetAsync(cand, 0, sizeof(uint32_t) * P * W, s->stream));
      unsigned long long total = 0;
      if (nq) {
        k_frontier_degrees<<<grid_for(nq, 256), 256, 0, s->stream>>>(queue, nq, s->off, deg);
        GRE_CUDA(cub::DeviceScan::ExclusiveSum(cubtmp, cubbytes, deg, prefix, nq + 1, s->stream));
        GRE_CUDA(cudaMemcpyAsync(&total, prefix + nq, sizeof total, cudaMemcpyDeviceToHost, s->stream));
        GRE_CUDA(cudaStreamSynchronize(s->stream));
        if (total) {
          const int grid = (int)std::min<uint64_t>((total + 255) / 256, (uint64_t)sms * 16);
          k_part_expand<<<grid, 256, 0, s->stream>>>(queue, nq, prefix, total, s->off, s->col, cand);
        }
        GRE_LAUNCH_CHECK();
      }
      GRE_CUDA(cudaMemcpyAsync(&c->scanned, &total, sizeof total, cudaMemcpyHostToDevice, s->stream));
      GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLTOALL, cand, recv, 4 * W));
      k_part_claim<<<grid_for(W, 256), 256, 0, s->stream>>>(W, P, recv, vis, lvl, d + 1, s->outdeg, nqueue, c);
      GRE_LAUNCH_CHECK();
      std::swap(queue, nqueue);
      bytes += 16 * nq + 8 * total + 4 * P * W * 3;
    } else {
      k_bu_step<<<grid_for(W * 32, 256, 8), 256, 0, s->stream>>>(L, s->roff, s->rcol, s->off, front_all, next, vis, lvl, d + 1, c);
      GRE_LAUNCH_CHECK();
      GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, next, front_all, 4 * W));
      std::swap(front, next);
    }
    GRE_CHECK(exchange_counters(p, xchg, ctx, c, call, &sum, &mine));
    if (bottom_up) bytes += 16 * (L - std::min<uint64_t>(L, visited / P)) + (uint64_t)(4.125 * (double)mine.scanned) + 4 * P * W;
    nq = mine.next_count;
    nf = sum.next_count;
    mf = sum.next_arcs;
    mu -= (int64_t)mf;
    visited += nf;
    scanned_total += sum.scanned;
    ++d;
    stats_record(st, nf);
  }
  // reached edges (all ranks), then the levels of every slot in caller order
  GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), s->stream));
  k_part_reached<<<grid_for(L, 256), 256, 0, s->stream>>>(L, lvl, s->outdeg, &c->next_arcs);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(exchange_counters(p, xchg, ctx, c, call, &sum, nullptr));
  GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, lvl, lvl_all, 4 * L));
  k_part_out<int32_t><<<grid_for(P * L, 256), 256, 0, s->stream>>>(P * L, p->xmap, lvl_all, dout);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(finish_output(s, level, dout, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = (uint32_t)(d > 0 ? d - 1 : 0);
    st->arcs_traversed = scanned_total;
    st->traversed_edges = s->symmetric() ? sum.next_arcs / 2 : sum.next_arcs;
    st->algo_bytes = bytes;
  }
  return GRE_SUCCESS;
}

int gre_part_pagerank(gre_part p, int variant, double d, uint32_t iters, double* pr, gre_exchange_fn xchg, void* ctx,
                      gre_stats* st) {
  if (!p || !pr || !xchg) return GRE_NULL;
  if ((variant != GRE_PR_REFERENCE && variant != GRE_PR_ITER) || !(d >= 0.0 && d < 1.0)) return GRE_INVALID_ARG;
  gre_graph s = p->sub;
  GRE_CHECK(use_graph(s));
  stats_reset(st);
  const uint64_t n = p->n, P = p->nparts, L = p->L;
  double *prl, *pr_all, *contrib, *contrib_all, *partial, *dout;
  GRE_CHECK(ws_array(s, WS_A, L, &prl));
  GRE_CHECK(ws_array(s, WS_B, P * L, &pr_all));
  GRE_CHECK(ws_array(s, WS_C, L, &contrib));
  GRE_CHECK(ws_array(s, WS_D, P * L, &contrib_all));
  GRE_CHECK(ws_array(s, WS_E, s->bins_in.n_partials + 1, &partial));
  GRE_CHECK(prepare_output(s, pr, n, WS_OUTBUF, &dout));
  const double tele = 1.0 - d;
  const bool refresh = variant == GRE_PR_ITER;
  RunTimer timer(s);
  k_part_pr_init<<<grid_for(L, 256), 256, 0, s->stream>>>(L, s->outdeg, tele, prl, contrib);
  GRE_LAUNCH_CHECK();
  for (uint32_t it = 0; it < iters; ++it) {
    // scatter-sync: every rank reads the contributions of all slots (fixed in the reference
    // variant: gathered once)
    if (it == 0 || refresh) GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, contrib, contrib_all, 8 * L));
    GRE_CHECK(rows::reduce_rows(s->bins_in, s->roff, PartGather{s->rcol, contrib_all},
                                PartFinish{prl, refresh ? contrib : nullptr, s->outdeg, tele, d}, partial, s->stream));
  }
  GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, prl, pr_all, 8 * L));
  k_part_out<double><<<grid_for(P * L, 256), 256, 0, s->stream>>>(P * L, p->xmap, pr_all, dout);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(finish_output(s, pr, dout, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = iters;
    for (uint32_t i = 0; i < iters; ++i) stats_record(st, rows::nonempty_rows(s->bins_in));
    st->arcs_traversed = p->arcs_in * (uint64_t)iters;  // this rank's in-arcs
    st->traversed_edges = p->m * (uint64_t)iters;
    // this rank: offsets, columns, gathered contributions, outdeg, pr and contribution writes,
    // plus the P * L contributions received
    st->algo_bytes = (8 * (L + 1) + 12 * p->arcs_in + 20 * L + 8 * P * L) * (uint64_t)iters;
  }
  return GRE_SUCCESS;
}

// A light superstep's offers travel as per-owner lists when (its most offers + 1) * d <= L, d from
// GRE_PART_SPARSE (default 8: lists of at most an eighth of the dense exchange's bytes); 0 keeps
// the dense exchange for every superstep.
static uint64_t part_sparse_offers() {
  if (const char* e = getenv("GRE_PART_SPARSE")) return strtoull(e, nullptr, 10);
  return 8;
}

int gre_part_sssp(gre_part p, uint32_t src, uint32_t* dist, gre_exchange_fn xchg, void* ctx, gre_stats* st) {
  if (!p || !dist || !xchg) return GRE_NULL;
  gre_graph s = p->sub;
  GRE_CHECK(use_graph(s));
  stats_reset(st);
  const uint64_t n = p->n, P = p->nparts, L = p->L, W = L / 32, me = p->rank;
  if (!p->w32) {
    set_error("gre_part_sssp: the graph had no uint32 weights when the part was made");
    return GRE_INVALID_ARG;
  }
  if (src >= n) {
    set_error("gre_part_sssp: source %u out of range (n = %llu)", src, (unsigned long long)n);
    return GRE_INVALID_ARG;
  }
  // the light/heavy split of the owned out-rows (once per part; delta is the whole graph's)
  const uint32_t delta = p->delta;
  if (delta && !p->sp_lend) {
    GRE_CUDA(cudaMalloc(&p->sp_col, sizeof(uint32_t) * (p->arcs_out ? p->arcs_out : 1)));
    GRE_CUDA(cudaMalloc(&p->sp_w, sizeof(uint32_t) * (p->arcs_out ? p->arcs_out : 1)));
    GRE_CUDA(cudaMalloc(&p->sp_lend, sizeof(uint64_t) * L));
    GRE_CHECK(sssp_split_rows(s->stream, L, s->off, s->col, p->w32, delta, p->sp_col, p->sp_w, p->sp_lend));
  }
  const uint64_t* off = s->off;
  const uint64_t* lend = delta ? p->sp_lend : s->off + 1;  // end of each row's light arcs
  const uint32_t* col = delta ? p->sp_col : s->col;
  const uint32_t* w = delta ? p->sp_w : p->w32;
  const DegreeBins* pB = nullptr;  // the part's rows binned as the one-GPU SSSP bins them
  GRE_CHECK(sssp_bins(s, s->roff == s->off, &pB));
  const DegreeBins& B = *pB;
  uint32_t *dl, *dist_all, *queue, *pend, *inb, *inb_all, *cand, *recv, *dout;
  uint64_t *deg, *prefix;
  SsspCounters *c, *call;
  BfsCounters *bc, *bcall;
  GRE_CHECK(ws_array(s, WS_A, L, &dl));
  GRE_CHECK(ws_array(s, WS_B, P * L, &dist_all));
  GRE_CHECK(ws_array(s, WS_C, W, &pend));
  uint32_t* farb;  // the far set: slots at or above the limit, examined again when it rises
  GRE_CHECK(ws_array(s, WS_N, W, &farb));
  GRE_CHECK(ws_array(s, WS_D, L, &queue));
  GRE_CHECK(ws_array(s, WS_F, W, &inb));
  GRE_CHECK(ws_array(s, WS_G, P * W, &inb_all));
  GRE_CHECK(ws_array(s, WS_I, P * L, &cand));
  uint32_t* touched;  // offer slots written since the last clear
  GRE_CHECK(ws_array(s, WS_H, P * W, &touched));
  GRE_CHECK(ws_array(s, WS_J, P * L, &recv));
  uint32_t* lists;  // per-owner offer lists of a light superstep (send side)
  GRE_CHECK(ws_array(s, WS_M, P * L, &lists));
  GRE_CHECK(ws_array(s, WS_K, L + 1, &deg));
  GRE_CHECK(ws_array(s, WS_L, L + 1, &prefix));
  uint32_t *tstart, *err;
  GRE_CHECK(ws_array(s, WS_E, p->arcs_out / sssp_tile_arcs() + 2, &tstart));
  GRE_CHECK(ws_array(s, WS_COUNTERS, 4, &c));  // c[0] counters, c[1] BFS-style totals, c[2] flags, c[3] pull counts
  GRE_CHECK(ws_array(s, WS_OUTBUF2, P, &call));
  bc = (BfsCounters*)(c + 1);
  err = (uint32_t*)(c + 2);
  unsigned long long* pull_counts = (unsigned long long*)(c + 3);  // arcs scanned, hits
  bcall = (BfsCounters*)call;
  GRE_CHECK(prepare_output(s, dist, n, WS_OUTBUF, &dout));
  void* cubtmp = nullptr;
  size_t cubbytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cubbytes, deg, prefix, L + 1, s->stream);
  GRE_CHECK(s->ws.get(WS_CUB, cubbytes, &cubtmp));
  const uint64_t bdiv = sssp_binned_divisor();
  const bool pull = p->w_sym && delta && sssp_pull_enabled();
  const uint64_t sparse = part_sparse_offers();
  const uint64_t pdiv = sssp_pull_arcs_divisor();

  RunTimer timer(s);
  uint32_t xr = 0;
  GRE_CUDA(cudaMemcpyAsync(&xr, p->xof + src, sizeof xr, cudaMemcpyDeviceToHost, s->stream));
  GRE_CUDA(cudaMemsetAsync(dl, 0xff, sizeof(uint32_t) * L, s->stream));
  GRE_CUDA(cudaMemsetAsync(pend, 0, sizeof(uint32_t) * W, s->stream));
  GRE_CUDA(cudaMemsetAsync(farb, 0, sizeof(uint32_t) * W, s->stream));
  GRE_CUDA(cudaMemsetAsync(inb, 0, sizeof(uint32_t) * W, s->stream));
  GRE_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), s->stream));
  GRE_CUDA(cudaMemsetAsync(pull_counts, 0, 2 * sizeof(unsigned long long), s->stream));
  GRE_CUDA(cudaMemsetAsync(cand, 0xff, sizeof(uint32_t) * P * L, s->stream));  // then cleared slot by slot
  GRE_CUDA(cudaMemsetAsync(touched, 0, sizeof(uint32_t) * P * W, s->stream));
  // Known distances of the other ranks' slots: upper bounds that let the relaxations drop offers
  // that cannot improve, as of the last all-gather of the distances (the pulled heavy passes make
  // one).  This rank's own heads are relaxed in place (OwnHeads), against its current distances.
  uint32_t* known = dist_all;
  GRE_CUDA(cudaMemsetAsync(known, 0xff, sizeof(uint32_t) * P * L, s->stream));
  OwnHeads own;
  own.lo = me * L;
  own.len = L;
  own.dist = dl;
  own.pend = pend;
  own.outdeg = s->outdeg;
  GRE_CUDA(cudaStreamSynchronize(s->stream));
  if (xr / L == me) {
    const uint32_t slot = xr - (uint32_t)(me * L), zero = 0, bit = 1u << (slot & 31u);
    GRE_CUDA(cudaMemcpyAsync(dl + slot, &zero, sizeof zero, cudaMemcpyHostToDevice, s->stream));
    GRE_CUDA(cudaMemcpyAsync(pend + (slot >> 5), &bit, sizeof bit, cudaMemcpyHostToDevice, s->stream));
  }
  // Supersteps of the reference's SSSP (every improved vertex scatters dist + w, combine = min),
  // ordered as the one-GPU path: pending slots below a global limit relax their light arcs (offers
  // to the owners: an all-to-all); when no rank has any left, the bucket's heavy arcs are relaxed
  // once (pulled by the slots at or above the limit from all-gathered distances and bucket bits
  // where the weights are symmetric, else offered); then the limit moves to the smallest pending
  // distance + delta.
  const uint32_t width = delta ? delta : 0xffffffffu;
  uint32_t limit = width;
  uint64_t relaxed = 0, bytes = 0, bucket = 0, bucket_heavy = 0;
  uint32_t steps = 0;
  std::vector<SsspCounters> h(P);
  // offers of this rank's frontier `list` (or bitmap `front`, binned form) over the light or heavy
  // ranges, exchanged with the owners, who keep the smallest and mark improved slots pending
  // `cap` > 0: every rank's offers of this pass are at most cap, and they travel as per-owner
  // (slot, distance) lists of cap pairs instead of the dense P * L offer arrays
  auto offer_pass = [&](const uint32_t* list, uint64_t nlist, const uint32_t* front, uint64_t arcs, bool heavy,
                        uint64_t cap) -> int {
    if (nlist && arcs && bdiv && nlist >= L / bdiv) {
      uint32_t* bits = const_cast<uint32_t*>(front);
      if (!bits) {  // the frontier as a bitmap, in the scan buffer (unused by this form)
        bits = (uint32_t*)deg;
        GRE_CUDA(cudaMemsetAsync(bits, 0, sizeof(uint32_t) * W, s->stream));
        k_queue_to_bits<<<grid_for(nlist, 256), 256, 0, s->stream>>>(list, nlist, bits);
        bytes += 4 * W + 4 * nlist;
      }
      GRE_CHECK(sssp_relax_binned_offer(s->stream, B, bits, off, lend, heavy, col, w, dl, cand, touched, known, own, nullptr));
      bytes += 16 * L + W * 4;  // rows scanned and their frontier bits (arcs below)
    } else if (nlist && arcs) {
      k_part_range_degrees<<<grid_for(nlist, 256), 256, 0, s->stream>>>(list, nlist, off, lend, heavy, deg);
      GRE_CUDA(cub::DeviceScan::ExclusiveSum(cubtmp, cubbytes, deg, prefix, nlist + 1, s->stream));
      GRE_CHECK(sssp_relax_tiles(s->stream, list, nlist, prefix, arcs, tstart, heavy ? lend : off, col, w, dl, cand, touched,
                                 err, known, own));
      bytes += 16 * nlist;
    }
    if (P == 1) {  // every head is this rank's own, relaxed in place: nothing was offered
      bytes += 12 * arcs;
    } else if (cap) {
      const uint64_t block = cap + 1;  // uint2: the count, then the pairs
      uint2* send = (uint2*)lists;
      GRE_CUDA(cudaMemset2DAsync(send, 8 * block, 0, 8, P, s->stream));
      const dim3 grid((unsigned)std::min<uint64_t>(grid_for(W, 256), 4 * 148), (unsigned)P);
      k_part_offers_pack<<<grid, 256, 0, s->stream>>>(W, touched, cand, send, block, cap, err);
      GRE_LAUNCH_CHECK();
      GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLTOALL, send, recv, 8 * block));
      k_part_sssp_claim_lists<<<grid_for(cap, 256, 4), 256, 0, s->stream>>>(P, L, (const uint2*)recv, block, cap, dl,
                                                                             s->outdeg, pend, err);
      bytes += 12 * arcs + 4 * P * W + 8 * P * block * 2;
    } else {
      GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLTOALL, cand, recv, 4 * L));
      k_part_offers_clear<<<grid_for(P * W, 256), 256, 0, s->stream>>>(P * W, touched, cand);  // after the exchange read cand
      k_part_sssp_claim<<<grid_for(L, 256), 256, 0, s->stream>>>(L, P, recv, dl, s->outdeg, pend);
      bytes += 12 * arcs + 4 * P * L * 2 + 4 * P * W + 4 * L;
    }
    GRE_LAUNCH_CHECK();
    relaxed += arcs;
    return GRE_SUCCESS;
  };
  bool rescan = false;                 // the limit rose: examine the far set again
  unsigned long long far_floor = ~0ull;  // this rank's smallest far distance seen so far
  for (;;) {
    // pageable: staged before the call returns
    const SsspCounters zero{0, 0, rescan ? 0xffffffffffffffffull : far_floor, 0, 0, 0, {0, 0}};
    GRE_CUDA(cudaMemcpyAsync(c, &zero, sizeof zero, cudaMemcpyHostToDevice, s->stream));
    k_part_sssp_select<<<grid_for(W, 256), 256, 0, s->stream>>>(W, pend, farb, rescan, dl, limit, off, lend, inb, queue, c);
    GRE_LAUNCH_CHECK();
    GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, c, call, sizeof(SsspCounters)));
    GRE_CUDA(cudaMemcpyAsync(h.data(), call, sizeof(SsspCounters) * P, cudaMemcpyDeviceToHost, s->stream));
    GRE_CUDA(cudaStreamSynchronize(s->stream));
    rescan = false;
    far_floor = h[me].min_far;
    uint64_t near = 0, pending = 0, min_far = ~0ull;
    for (const SsspCounters& x : h) {
      near += x.near;
      pending += x.pending;
      bucket += x.bucket_new;
      bucket_heavy += x.heavy_new;
      min_far = std::min<uint64_t>(min_far, x.min_far);
    }
    bytes += 12 * W + 8 * h[me].near;  // pending, far and bucket words; the frontier's distances
    if (near) {  // a light superstep
      uint64_t most = 0;  // the most offers any rank can make (the same on every rank)
      for (const SsspCounters& x : h) most = std::max<uint64_t>(most, x.arcs);
      const uint64_t cap = sparse && (most + 1) * sparse <= L && 2 * (most + 1) <= L ? std::max<uint64_t>(most, 1) : 0;
      GRE_CHECK(offer_pass(queue, h[me].near, nullptr, h[me].arcs, false, cap));
      ++steps;
      stats_record(st, near);
      continue;
    }
    if (bucket) {  // the bucket is settled: its heavy arcs, once (every rank sees the same sums)
      // pulled when the bucket has many members or many heavy arcs (the same sums on every rank)
      if (pull && bdiv && (bucket >= P * L / bdiv || (pdiv && bucket_heavy * pdiv >= p->m))) {
        GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, dl, dist_all, 4 * L));
        GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, inb, inb_all, 4 * W));
        GRE_CHECK(sssp_pull_binned(s->stream, B, inb_all, off, lend, true, col, w, dist_all, dl, pend, limit, pull_counts));
        bytes += 4 * P * L + 4 * P * W + 16 * L;
      } else {
        uint64_t nb = 0, arcs = 0;
        {  // this rank's members as a queue (for the tiles) and the count of their heavy arcs
          unsigned long long* cnt = (unsigned long long*)&bc->next_count;
          GRE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s->stream));
          k_bits_to_queue<<<grid_for(W, 256), 256, 0, s->stream>>>(L, inb, queue, cnt);
          GRE_LAUNCH_CHECK();
          unsigned long long hn = 0;
          GRE_CUDA(cudaMemcpyAsync(&hn, cnt, sizeof hn, cudaMemcpyDeviceToHost, s->stream));
          GRE_CUDA(cudaStreamSynchronize(s->stream));
          nb = hn;
          if (nb) {
            k_part_range_degrees<<<grid_for(nb, 256), 256, 0, s->stream>>>(queue, nb, off, lend, true, deg);
            GRE_CUDA(cub::DeviceScan::ExclusiveSum(cubtmp, cubbytes, deg, prefix, nb + 1, s->stream));
            GRE_CUDA(cudaMemcpyAsync(&arcs, prefix + nb, sizeof arcs, cudaMemcpyDeviceToHost, s->stream));
            GRE_CUDA(cudaStreamSynchronize(s->stream));
          }
        }
        GRE_CHECK(offer_pass(queue, nb, inb, arcs, true, 0));
      }
      GRE_CUDA(cudaMemsetAsync(inb, 0, sizeof(uint32_t) * W, s->stream));
      bucket = 0;
      bucket_heavy = 0;
      ++steps;
      stats_record(st, 0);
      continue;
    }
    if (pending == 0) break;
    // every rank sees the same sums: the same new limit.  min_far is exact after a rescan and a
    // lower bound otherwise (a far slot that later left the set may have set it): a rescan that
    // brings nothing below the new limit computes the exact value for the next rise.
    limit = min_far > 0xffffffffull - width ? 0xffffffffu : (uint32_t)(min_far + width);
    rescan = true;
  }
  GRE_CUDA(cudaMemsetAsync(bc, 0, sizeof(BfsCounters), s->stream));
  k_part_reached_dist<<<grid_for(L, 256), 256, 0, s->stream>>>(L, dl, s->outdeg, &bc->next_arcs);
  GRE_LAUNCH_CHECK();
  BfsCounters sum;
  GRE_CHECK(exchange_counters(p, xchg, ctx, bc, bcall, &sum, nullptr));
  GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, dl, dist_all, 4 * L));
  k_part_out<uint32_t><<<grid_for(P * L, 256), 256, 0, s->stream>>>(P * L, p->xmap, dist_all, dout);
  GRE_LAUNCH_CHECK();
  // checked after the last collective, so that every rank takes the same ones
  uint32_t herr = 0;
  unsigned long long pc[2] = {0, 0};
  GRE_CUDA(cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, s->stream));
  GRE_CUDA(cudaMemcpyAsync(pc, pull_counts, sizeof pc, cudaMemcpyDeviceToHost, s->stream));
  GRE_CUDA(cudaStreamSynchronize(s->stream));
  if (herr) {
    set_error(herr & 1u ? "gre_part_sssp: frontier tile overflow" : "gre_part_sssp: offer list overflow");
    return GRE_FAILURE;
  }
  GRE_CHECK(finish_output(s, dist, dout, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = steps;
    st->arcs_traversed = relaxed + pc[0];  // this rank's
    st->traversed_edges = s->symmetric() ? sum.next_arcs / 2 : sum.next_arcs;
    st->algo_bytes = bytes + 4 * pc[0] + 8 * pc[1];
  }
  return GRE_SUCCESS;
}

int gre_part_cc(gre_part p, uint32_t* label, gre_exchange_fn xchg, void* ctx, gre_stats* st) {
  if (!p || !label || !xchg) return GRE_NULL;
  gre_graph s = p->sub;
  GRE_CHECK(use_graph(s));
  stats_reset(st);
  const uint64_t n = p->n, P = p->nparts, L = p->L, me = p->rank;
  const uint32_t lo = (uint32_t)(me * L);
  const bool sym = s->roff == s->off;
  const uint32_t* key = p->xmap + me * L;  // caller id of every owned slot (padding: 0xffffffff)
  uint32_t *lab, *lab_all, *dout, *parent, *rootlab, *skip;
  double* partial;
  BfsCounters *c, *call;
  constexpr uint32_t kSampled = 2, kSample = 1024;
  GRE_CHECK(ws_array(s, WS_A, L, &lab));
  GRE_CHECK(ws_array(s, WS_B, P * L, &lab_all));
  GRE_CHECK(ws_array(s, WS_C, L, &parent));
  GRE_CHECK(ws_array(s, WS_D, L, &rootlab));
  GRE_CHECK(ws_array(s, WS_E, ((L + 31) >> 5) + kSample, &skip));
  GRE_CHECK(ws_array(s, WS_F, std::max(s->bins_in.n_partials, s->bins_out.n_partials) + 1, &partial));
  GRE_CHECK(ws_array(s, WS_COUNTERS, 2, &c));
  GRE_CHECK(ws_array(s, WS_OUTBUF2, P, &call));
  GRE_CHECK(prepare_output(s, label, n, WS_OUTBUF, &dout));
  unsigned long long* counts = (unsigned long long*)(c + 1);  // Afforest's arc counts (byte model)
  uint32_t* sample = skip + ((L + 31) >> 5);
  if (p->cc_remote == ~0ull) {  // once per part: arcs that cross to other ranks
    GRE_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned long long), s->stream));
    k_pcc_count_remote<<<grid_for(p->arcs_in, 256, 8), 256, 0, s->stream>>>(p->arcs_in, s->rcol, lo, (uint32_t)L, counts);
    if (!sym) k_pcc_count_remote<<<grid_for(p->arcs_out, 256, 8), 256, 0, s->stream>>>(p->arcs_out, s->col, lo, (uint32_t)L, counts);
    GRE_LAUNCH_CHECK();
    unsigned long long h = 0;
    GRE_CUDA(cudaMemcpyAsync(&h, counts, sizeof h, cudaMemcpyDeviceToHost, s->stream));
    GRE_CUDA(cudaStreamSynchronize(s->stream));
    p->cc_remote = h;
  }
  RunTimer timer(s);
  // phase 1: union-find over the arcs inside this rank (Afforest on a symmetric graph, as gre_cc:
  // the first arcs of every row, then the rows outside the largest local component)
  uint64_t visited = 0;
  k_uf_init<<<grid_for(L, 256), 256, 0, s->stream>>>(L, parent);
  if (sym) {
    k_pcc_sample<<<grid_for(L, 256), 256, 0, s->stream>>>(L, s->roff, s->rcol, kSampled, lo, parent, key);
    const uint64_t stride = L > kSample ? L / kSample : 1;
    const uint32_t ns = (uint32_t)std::min<uint64_t>(kSample, (L + stride - 1) / stride);
    k_uf_compress<<<grid_for(L, 256), 256, 0, s->stream>>>(L, parent, stride, sample, ns);
    std::vector<uint32_t> hs(kSample, 0);
    GRE_CUDA(cudaMemcpyAsync(hs.data(), sample, sizeof(uint32_t) * ns, cudaMemcpyDeviceToHost, s->stream));
    GRE_CUDA(cudaStreamSynchronize(s->stream));
    const uint32_t big = uf_most_frequent(hs, ns);
    GRE_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), s->stream));
    k_uf_skipbits<<<grid_for((L + 31) >> 5, 256), 256, 0, s->stream>>>(L, parent, s->roff, big, kSampled, skip, counts);
    HookLocal rest{s->rcol, parent, key, lo, (uint32_t)L, skip, s->roff, kSampled};
    GRE_CHECK(rows::reduce_rows(s->bins_in, s->roff, rest, NoFinishPart{}, partial, s->stream));
    unsigned long long h[2] = {0, 0};
    GRE_CUDA(cudaMemcpyAsync(h, counts, sizeof h, cudaMemcpyDeviceToHost, s->stream));
    GRE_CUDA(cudaStreamSynchronize(s->stream));
    visited = h[0] + h[1];
  } else {  // weak components: in-arcs and out-arcs
    GRE_CHECK(rows::reduce_rows(s->bins_in, s->roff, HookLocal{s->rcol, parent, key, lo, (uint32_t)L}, NoFinishPart{}, partial,
                                s->stream));
    GRE_CHECK(rows::reduce_rows(s->bins_out, s->off, HookLocal{s->col, parent, key, lo, (uint32_t)L}, NoFinishPart{}, partial,
                                s->stream));
    visited = p->arcs_in + p->arcs_out;
  }
  k_uf_compress<<<grid_for(L, 256), 256, 0, s->stream>>>(L, parent, L + 1, nullptr, 0);
  k_pcc_labels<<<grid_for(L, 256), 256, 0, s->stream>>>(L, parent, key, lab, rootlab);
  GRE_LAUNCH_CHECK();
  uint64_t bytes = 8 * (L + 1) + 12 * visited + 16 * L;
  // phase 2: the local components' labels meet over the cut arcs, a round per all-gather of the
  // labels; each round also takes the shortcut through the vertex a label names.  Every rank
  // takes the same collectives (a rank without cut arcs still exchanges).
  auto cut_sweep = [&](const DegreeBins& B, const uint64_t* off, const uint32_t* col) {
    auto lanes = [&](auto kernel, int b, int G) {
      if (B.count[b])
        kernel<<<grid_for(B.count[b] * G, 256, 8), 256, 0, s->stream>>>(B.rows + B.start[b], B.count[b], off, col, lo,
                                                                          (uint32_t)L, lab_all, parent, rootlab);
    };
    lanes(k_pcc_cut_lanes<1>, 0, 1);
    lanes(k_pcc_cut_lanes<2>, 1, 2);
    lanes(k_pcc_cut_lanes<4>, 2, 4);
    lanes(k_pcc_cut_lanes<8>, 3, 8);
    lanes(k_pcc_cut_lanes<16>, 4, 16);
    lanes(k_pcc_cut_lanes<32>, 5, 32);
    const uint64_t nbig = B.count[6] + B.count[7];
    if (nbig)
      k_pcc_cut_rows<<<grid_for(nbig * 256, 256, 8), 256, 0, s->stream>>>(B.rows + B.start[6], nbig, off, col, lo, (uint32_t)L,
                                                                            lab_all, parent, rootlab);
  };
  uint32_t steps = 0;
  BfsCounters sum;
  for (;;) {
    GRE_CHECK(exchange(p, xchg, ctx, GRE_XCHG_ALLGATHER, lab, lab_all, 4 * L));
    GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), s->stream));
    if (p->cc_remote) {
      cut_sweep(s->bins_in, s->roff, s->rcol);
      if (!sym) cut_sweep(s->bins_out, s->off, s->col);
      bytes += 4 * (p->arcs_in + (sym ? 0 : p->arcs_out)) + 4 * p->cc_remote;
    }
    k_pcc_roots<<<grid_for(L, 256), 256, 0, s->stream>>>(L, parent, lab_all, p->xof, rootlab);
    k_pcc_members<<<grid_for(L, 256), 256, 0, s->stream>>>(L, parent, rootlab, lab, c);
    GRE_LAUNCH_CHECK();
    GRE_CHECK(exchange_counters(p, xchg, ctx, c, call, &sum, nullptr));
    ++steps;
    bytes += 4 * P * L + 16 * L;
    stats_record(st, sum.next_count);
    if (sum.next_count == 0) break;
  }
  k_part_out<uint32_t><<<grid_for(P * L, 256), 256, 0, s->stream>>>(P * L, p->xmap, lab_all, dout);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(finish_output(s, label, dout, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = steps;
    st->arcs_traversed = visited + (uint64_t)steps * (p->cc_remote ? p->arcs_in + (sym ? 0 : p->arcs_out) : 0);
    st->traversed_edges = s->symmetric() ? p->m / 2 : p->m;
    st->algo_bytes = bytes;
  }
  return GRE_SUCCESS;
}

}  // extern "C"
