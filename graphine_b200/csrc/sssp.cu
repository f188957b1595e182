// SSSP fast path: near-far frontier relaxation with uint32 weights.
//
// Same fixed point as the reference SSSP plugin (Kernels/SSSP.hpp:55-89: scatter last[u]+w,
// combine = min, every improved vertex re-activated): shortest-path distances are unique, so
// the result is bit-exact whatever the relaxation order.  Differences from the reference's
// superstep, chosen for the GPU:
//   * near-far ordering (Davidson et al., IPDPS 2014): improved vertices below a moving limit
//     form the next frontier, the others wait in a far set until the limit (raised by a bucket
//     width delta, or to the smallest waiting distance + delta) passes them; with the light/heavy
//     split of delta-stepping (Meyer and Sanders 2003) only arcs lighter than delta are relaxed
//     inside a bucket and a settled bucket's heavy arcs once.  On RMAT this relaxes each arc
//     about 1.1 times instead of about 2.2 for a plain Bellman-Ford frontier (delta = 0);
//   * the frontier is expanded edge-balanced in tiles of 2048 consecutive frontier arcs (the
//     owners staged in shared memory, owner of each arc by a block max-scan), so hubs do not
//     serialise a warp;
//   * an improvement is a fire-and-forget atomic min on the distance plus a bit in a changed
//     bitmap: no thread waits for an atomic's reply (hub heads receive thousands per superstep),
//     and a pass over the bitmap builds the next frontier and far set without duplicates;
//   * the far set is a bitmap: a limit rise scans it, reading the far vertices' distances in
//     vertex order, 32 to a word (against a list of far vertices, read at random: RMAT-26 SSSP
//     18.5 -> 17.8 ms);
//   * the distance of a frontier vertex is read when its tile starts (not a copy taken at the
//     start of the superstep), which can only lower the values sent;
//   * vertices without out-arcs are never queued (they have nothing to relax).
//
// Byte model per superstep: 16 F (queue + offsets) + 12 A (column + weight + dist probe)
// + 8 N (queue append + bitmap), F frontier, A arcs relaxed, N improved vertices.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>

#include "gre_internal.cuh"

namespace gre {

// defined in bfs.cu
__global__ void k_queue_to_bits(const uint32_t* __restrict__ queue, uint64_t nq, uint32_t* __restrict__ bits);

template <class T>
static int ws_array(gre_graph g, int slot, uint64_t count, T** p) {
  void* v = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &v));
  *p = (T*)v;
  return GRE_SUCCESS;
}


// Arc counts of the queued vertices in the range being relaxed (light: [off[v], lend[v]),
// heavy: [lend[v], off[v+1])), for the scan.
template <bool HEAVY>
__global__ void k_sssp_degrees(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ off,
                               const uint64_t* __restrict__ lend, uint64_t* __restrict__ deg) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = queue[i];
    deg[i] = HEAVY ? off[v + 1] - lend[v] : lend[v] - off[v];
  }
}

// Light/heavy split of each row for bucket width delta (warp per row, stable within a class).
__global__ void k_split_light_heavy(uint64_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                                    const uint32_t* __restrict__ w, uint32_t delta, uint32_t* __restrict__ ocol,
                                    uint32_t* __restrict__ ow, uint64_t* __restrict__ lsplit) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t below = (1u << lane) - 1u;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint64_t a0 = off[v], a1 = off[v + 1];
    uint64_t nlight = 0;
    for (uint64_t b = a0; b < a1; b += 32) {
      const bool light = b + lane < a1 && w[b + lane] < delta;
      nlight += __popc(__ballot_sync(0xffffffffu, light));
    }
    uint64_t lc = a0, hc = a0 + nlight;
    for (uint64_t b = a0; b < a1; b += 32) {
      const bool in = b + lane < a1;
      const uint32_t x = in ? w[b + lane] : 0u;
      const bool light = in && x < delta;
      const uint32_t lm = __ballot_sync(0xffffffffu, light);
      const uint32_t hm = __ballot_sync(0xffffffffu, in && !light);
      if (in) {
        const uint64_t dst = light ? lc + __popc(lm & below) : hc + __popc(hm & below);
        ocol[dst] = col[b + lane];
        ow[dst] = x;
      }
      lc += __popc(lm);
      hc += __popc(hm);
    }
    if (lane == 0) lsplit[v] = a0 + nlight;
  }
}

// Edge-balanced expansion in tiles of kTile consecutive frontier arcs.  k_tile_starts records,
// for every tile, the frontier index owning its first arc (each frontier vertex writes the
// tiles that begin inside its arc range, so every entry is written exactly once).  A CTA then
// stages the owners of its tile (at most kTile + 1 of them, since queued vertices have at least
// one out-arc) in shared memory and each thread finds the owner of its arc there: the per-arc
// search touches shared memory only, and the column and weight reads of one vertex coalesce.
// Queue appends are gathered per tile in shared memory and reserved with one global atomic per
// tile, so the queue counters are not a point of contention.
constexpr int kTileThreads = 256;
constexpr int kTileItems = 8;
constexpr uint64_t kTile = (uint64_t)kTileThreads * kTileItems;
static_assert(kTileItems == 8, "owner scan packs 8 uint16 per thread");

struct MaxOp {
  __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

__global__ void k_tile_starts(const uint64_t* __restrict__ prefix, uint64_t nq, uint32_t* __restrict__ start) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p0 = prefix[i], p1 = prefix[i + 1];
    if (p1 == p0) continue;
    for (uint64_t t = (p0 + kTile - 1) / kTile; t <= (p1 - 1) / kTile; ++t) start[t] = (uint32_t)i;
  }
}

// Offer forms: an arc to head x offering nd.  A head in `own` is relaxed in place (its distance
// probed, lowered by atomic min, its pending bit set when it has out-arcs); another head is
// probed against known[x] (when given) and the offer array, and offered by atomic min with its
// bit in `touched`.  probe() returns the value nd must beat; commit() applies an offer that does.
struct OfferArc {
  uint64_t lx;
  bool mine;
  __device__ __forceinline__ uint32_t probe(const OwnHeads& o, const uint32_t* known, const uint32_t* offers, uint32_t x,
                                            uint32_t nd) {
    lx = (uint64_t)x - o.lo;
    mine = lx < o.len;
    if (mine) return __ldcg(o.dist + lx);
    if (known && nd >= __ldcg(known + x)) return 0u;
    return __ldcg(offers + x);
  }
  __device__ __forceinline__ void commit(const OwnHeads& o, uint32_t* offers, uint32_t* touched, uint32_t x, uint32_t nd) const {
    if (mine) {
      atomicMin(o.dist + lx, nd);
      if (o.outdeg[lx]) atomicOr(o.pend + (lx >> 5), 1u << (lx & 31u));
    } else {
      atomicMin(offers + x, nd);
      if (touched) atomicOr(touched + (x >> 5), 1u << (x & 31u));
    }
  }
};

// OFFER: the owners' distances come from srcdist and `dist` is a separate offer array (the
// partitioned path); otherwise from dist itself.  Either way an improved entry sets its bit in
// `changed` when that bitmap is given.
template <bool OFFER>
__global__ void __launch_bounds__(kTileThreads) k_sssp_relax(const uint32_t* __restrict__ queue, uint64_t nq,
                                                             const uint64_t* __restrict__ prefix, uint64_t total, const uint32_t* __restrict__ start,
                                                             const uint64_t* __restrict__ base, const uint32_t* __restrict__ col,
                                                             const uint32_t* __restrict__ w, const uint32_t* __restrict__ srcdist,
                                                             uint32_t* __restrict__ dist, uint32_t* __restrict__ changed,
                                                             uint32_t* __restrict__ error, const uint32_t* __restrict__ known,
                                                             const OwnHeads own) {
  using OwnerScan = cub::BlockScan<uint32_t, kTileThreads>;
  __shared__ uint64_t s_arc[kTile + 1];                // arc index at tile position s_rel[j]
  __shared__ uint32_t s_du[kTile + 1];                 // distance of owner j
  __shared__ uint16_t s_rel[kTile + 1];                // first tile position of owner j
  __shared__ __align__(16) uint16_t s_own[kTile];      // owner of each tile position
  __shared__ typename OwnerScan::TempStorage s_scan;
  const uint64_t ntiles = (total + kTile - 1) / kTile;
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint64_t t0 = tile * kTile;
    const uint32_t len = (uint32_t)(total - t0 < kTile ? total - t0 : kTile);
    const uint64_t lo = start[tile];
    const uint64_t hi = tile + 1 < ntiles ? start[tile + 1] : nq - 1;
    const uint64_t cnt = hi - lo + 1;
    if (cnt > kTile + 1) {  // cannot happen while every queued vertex has an out-arc; uniform
      if (threadIdx.x == 0) atomicOr(error, 1u);
      continue;
    }
    *(uint4*)(s_own + threadIdx.x * kTileItems) = make_uint4(0, 0, 0, 0);
    for (uint64_t j = threadIdx.x; j < cnt; j += kTileThreads) {
      const uint32_t u = queue[lo + j];
      const uint64_t p = prefix[lo + j];
      const uint64_t r = p > t0 ? p - t0 : 0;
      s_rel[j] = (uint16_t)r;
      s_arc[j] = base[u] + (t0 + r - p);
      s_du[j] = __ldcg((OFFER ? srcdist : dist) + u);
    }
    __syncthreads();
    // owner of every tile position: mark where each owner's arcs begin, then a running maximum
    // (owners begin at strictly increasing positions, every queued vertex having an out-arc)
    for (uint32_t j = 1 + threadIdx.x; j < cnt; j += kTileThreads)
      if (s_rel[j] < len) s_own[s_rel[j]] = (uint16_t)j;
    __syncthreads();
    {
      uint32_t own[kTileItems];
      const uint4 raw = *(const uint4*)(s_own + threadIdx.x * kTileItems);
      const uint32_t wds[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        own[2 * k] = wds[k] & 0xffffu;
        own[2 * k + 1] = wds[k] >> 16;
      }
      OwnerScan(s_scan).InclusiveScan(own, own, MaxOp());
      *(uint4*)(s_own + threadIdx.x * kTileItems) =
          make_uint4(own[0] | own[1] << 16, own[2] | own[3] << 16, own[4] | own[5] << 16, own[6] | own[7] << 16);
    }
    __syncthreads();
    // the thread's kTileItems arcs in rounds of independent loads (column and weight, then the
    // head's distance); an improvement is a fire-and-forget atomic min plus a bit in `changed`,
    // so no thread waits for an atomic's reply (hub heads receive many of them)
    uint32_t du[kTileItems], v[kTileItems], wt[kTileItems], dv[kTileItems];
#pragma unroll
    for (int k = 0; k < kTileItems; ++k) {
      const uint32_t t = (uint32_t)k * kTileThreads + threadIdx.x;
      const uint32_t a = s_own[t];
      const uint64_t arc = s_arc[a] + (t - s_rel[a]);
      du[k] = s_du[a];
      const bool ok = t < len;
      v[k] = ok ? __ldg(col + arc) : 0u;
      wt[k] = ok ? __ldg(w + arc) : 0u;
    }
    if (OFFER) {
      OfferArc oa[kTileItems];
#pragma unroll
      for (int k = 0; k < kTileItems; ++k) {
        const bool ok = (uint32_t)k * kTileThreads + threadIdx.x < len;
        dv[k] = ok ? oa[k].probe(own, known, dist, v[k], du[k] + wt[k]) : 0u;
      }
#pragma unroll
      for (int k = 0; k < kTileItems; ++k) {
        const uint32_t nd = du[k] + wt[k];
        if (nd < dv[k]) oa[k].commit(own, dist, changed, v[k], nd);
      }
    } else {
#pragma unroll
      for (int k = 0; k < kTileItems; ++k) {
        const bool ok = (uint32_t)k * kTileThreads + threadIdx.x < len;
        dv[k] = ok ? __ldcg(dist + v[k]) : 0u;
      }
#pragma unroll
      for (int k = 0; k < kTileItems; ++k) {
        const bool ok = (uint32_t)k * kTileThreads + threadIdx.x < len;
        const uint32_t nd = du[k] + wt[k];
        if (ok && nd < dv[k]) {
          atomicMin(dist + v[k], nd);
          if (changed) atomicOr(changed + (v[k] >> 5), 1u << (v[k] & 31u));
        }
      }
    }
    __syncthreads();
  }
}

// Large frontiers relaxed through the degree bins of the CSR instead of arc tiles: every bin's
// rows are scanned in order, and a row whose vertex is in the frontier bitmap relaxes its light
// ([off, lend)) or heavy ([lend, off+1)) arcs with 1..32 lanes (bins 0-5), a CTA (bin 6) or a CTA
// per 65536-arc chunk (bin 7).  No queue scan, no tile staging and no block barriers: the
// relaxations of a large frontier stream like the PageRank pull.  Same improvements (atomic min
// and a changed bit) as the tile kernel.
struct RelaxRange {
  const uint32_t* __restrict__ front;  // frontier bitmap
  const uint64_t* __restrict__ off;
  const uint64_t* __restrict__ lend;
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ w;
  uint32_t* __restrict__ dist;
  uint32_t* __restrict__ changed;
  unsigned long long* __restrict__ arcs;  // arcs relaxed (statistics)
  bool heavy;
  const uint32_t* __restrict__ srcdist;  // OFFER form: the rows' own distances (dist holds offers)
  const uint32_t* __restrict__ known;    // OFFER form: upper bounds of the heads' distances (may be null)
  OwnHeads oh;                           // OFFER form: heads relaxed in place
  __device__ __forceinline__ bool in(uint32_t v) const { return (__ldg(front + (v >> 5)) >> (v & 31u)) & 1u; }
  __device__ __forceinline__ void range(uint32_t v, uint64_t* lo, uint64_t* hi) const {
    *lo = heavy ? lend[v] : off[v];
    *hi = heavy ? off[v + 1] : lend[v];
  }
  // arcs a, a + step, ... < hi offered du + w; four column/weight loads, then four distance
  // probes in flight per lane.  OFFER: dist is a separate offer array, probed and committed as
  // OfferArc says.
  template <bool OFFER>
  __device__ __forceinline__ uint32_t own(uint32_t v) const { return __ldcg((OFFER ? srcdist : dist) + v); }
  template <bool OFFER>
  __device__ __forceinline__ void relax(uint32_t du, uint64_t a, uint64_t hi, uint64_t step) const {
    for (; a + 3 * step < hi; a += 4 * step) {
      uint32_t x[4], nd[4], dv[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        x[k] = __ldg(col + a + k * step);
        nd[k] = du + __ldg(w + a + k * step);
      }
      if (OFFER) {
        OfferArc oa[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) dv[k] = oa[k].probe(oh, known, dist, x[k], nd[k]);
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (nd[k] < dv[k]) oa[k].commit(oh, dist, changed, x[k], nd[k]);
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) dv[k] = __ldcg(dist + x[k]);
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (nd[k] < dv[k]) {
            atomicMin(dist + x[k], nd[k]);
            if (changed) atomicOr(changed + (x[k] >> 5), 1u << (x[k] & 31u));
          }
      }
    }
    for (; a < hi; a += step) {
      const uint32_t x = __ldg(col + a);
      const uint32_t nd = du + __ldg(w + a);
      if (OFFER) {
        OfferArc oa;
        if (nd < oa.probe(oh, known, dist, x, nd)) oa.commit(oh, dist, changed, x, nd);
      } else if (nd < __ldcg(dist + x)) {
        atomicMin(dist + x, nd);
        if (changed) atomicOr(changed + (x >> 5), 1u << (x & 31u));
      }
    }
  }
};

// c may be null (the caller counts the arcs another way)
__device__ __forceinline__ void add_arcs(unsigned long long* c, unsigned long long k) {
  for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
  if ((threadIdx.x & 31u) == 0 && k && c) atomicAdd(c, k);
}

template <int G, bool OFFER>
__global__ void __launch_bounds__(256) k_relax_lanes(const uint32_t* __restrict__ rows, uint64_t count, RelaxRange R) {
  const uint32_t lane = threadIdx.x & 31u, lig = lane % G;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long arcs = 0;
  for (uint64_t base = warp * (32 / G); base < count; base += nwarps * (32 / G)) {
    const uint64_t i = base + lane / G;
    if (i >= count) continue;
    const uint32_t v = rows[i];
    if (!R.in(v)) continue;
    uint64_t lo, hi;
    R.range(v, &lo, &hi);
    if (lo >= hi) continue;
    if (lig == 0) arcs += hi - lo;
    R.template relax<OFFER>(R.template own<OFFER>(v), lo + lig, hi, G);
  }
  add_arcs(R.arcs, arcs);
}

template <bool OFFER>
__global__ void __launch_bounds__(256) k_relax_cta(const uint32_t* __restrict__ rows, uint64_t count, RelaxRange R) {
  unsigned long long arcs = 0;
  for (uint64_t i = blockIdx.x; i < count; i += gridDim.x) {
    const uint32_t v = rows[i];
    if (!R.in(v)) continue;
    uint64_t lo, hi;
    R.range(v, &lo, &hi);
    if (threadIdx.x == 0 && hi > lo) arcs += hi - lo;
    R.template relax<OFFER>(R.template own<OFFER>(v), lo + threadIdx.x, hi, blockDim.x);
  }
  add_arcs(R.arcs, arcs);
}

// chunk c: arcs [chunk_begin[c], + chunk) of the row, cut to the light or heavy range
template <bool OFFER>
__global__ void __launch_bounds__(256) k_relax_chunks(const uint32_t* __restrict__ rows, const uint64_t* __restrict__ chunk_row,
                                                      const uint64_t* __restrict__ chunk_begin, uint64_t nchunks, uint64_t chunk,
                                                      RelaxRange R) {
  unsigned long long arcs = 0;
  for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const uint32_t v = rows[chunk_row[c]];
    if (!R.in(v)) continue;
    uint64_t lo, hi;
    R.range(v, &lo, &hi);
    const uint64_t c0 = chunk_begin[c], c1 = c0 + chunk;
    lo = lo > c0 ? lo : c0;
    hi = hi < c1 ? hi : c1;
    if (lo >= hi) continue;
    if (threadIdx.x == 0) arcs += hi - lo;
    R.template relax<OFFER>(R.template own<OFFER>(v), lo + threadIdx.x, hi, blockDim.x);
  }
  add_arcs(R.arcs, arcs);
}

template <bool OFFER>
static int relax_binned(const DegreeBins& B, const RelaxRange& R, cudaStream_t s) {
  const uint32_t* r = B.rows;
  auto grid = [](uint64_t threads) { return grid_for(threads, 256, 8); };
  if (B.count[0]) k_relax_lanes<1, OFFER><<<grid(B.count[0]), 256, 0, s>>>(r + B.start[0], B.count[0], R);
  if (B.count[1]) k_relax_lanes<2, OFFER><<<grid(B.count[1] * 2), 256, 0, s>>>(r + B.start[1], B.count[1], R);
  if (B.count[2]) k_relax_lanes<4, OFFER><<<grid(B.count[2] * 4), 256, 0, s>>>(r + B.start[2], B.count[2], R);
  if (B.count[3]) k_relax_lanes<8, OFFER><<<grid(B.count[3] * 8), 256, 0, s>>>(r + B.start[3], B.count[3], R);
  if (B.count[4]) k_relax_lanes<16, OFFER><<<grid(B.count[4] * 16), 256, 0, s>>>(r + B.start[4], B.count[4], R);
  if (B.count[5]) k_relax_lanes<32, OFFER><<<grid(B.count[5] * 32), 256, 0, s>>>(r + B.start[5], B.count[5], R);
  if (B.count[6]) k_relax_cta<OFFER><<<grid(B.count[6] * 256), 256, 0, s>>>(r + B.start[6], B.count[6], R);
  if (B.count[7])
    k_relax_chunks<OFFER><<<grid(B.n_hub_chunks * 256), 256, 0, s>>>(r + B.start[7], B.hub_chunk_row, B.hub_chunk_begin,
                                                                     B.n_hub_chunks, B.sched.hub_chunk, R);
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

// Pull form of a large pass (direction-optimising, as bottom-up BFS): instead of the frontier
// pushing along its arcs, every vertex that can still improve scans its own light (or heavy)
// arcs for neighbours in the frontier bitmap and takes the smallest dist[u] + w.  Valid when the
// graph is symmetric and w(u->v) == w(v->u) (g->w32_symmetric): v's arc to u then carries the
// weight, and the light/heavy class, of u's arc to v, so the candidate values are exactly those
// the push would offer.  What it saves: the push's reads and atomics land on the heads, spread
// over all of dist (DRAM); the pull reads dist only at frontier vertices (on RMAT mostly the
// hubs, which the degree-ordered ids keep in L2) and writes each improved vertex once.  Rows
// whose distance is below `lo` are settled (every earlier bucket is final) and are skipped
// after one read of dist.
struct PullRange {
  const uint32_t* __restrict__ front;  // sources: the near frontier (light pass) or the bucket (heavy pass)
  const uint64_t* __restrict__ off;
  const uint64_t* __restrict__ lend;
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ w;
  uint32_t* __restrict__ dist;               // the rows' distances (improved in place)
  uint32_t* __restrict__ changed;            // a bit per improved row
  unsigned long long* __restrict__ counts;  // [0] arcs scanned, [1] frontier hits
  bool heavy;
  uint32_t lo;
  const uint32_t* __restrict__ srcdist;      // the frontier's distances, indexed by column (the
                                             // one-GPU path: dist itself)
  __device__ __forceinline__ void range(uint32_t v, uint64_t* a0, uint64_t* a1) const {
    *a0 = heavy ? lend[v] : off[v];
    *a1 = heavy ? off[v + 1] : lend[v];
  }
  // smallest dist[u] + w over the arcs a, a + step, ... < hi whose tail u is in the frontier;
  // four column loads and bit tests in flight, then the hits' weights and distances
  __device__ __forceinline__ uint32_t best(uint64_t a, uint64_t hi, uint64_t step, unsigned long long* hits) const {
    uint32_t b = 0xffffffffu;
    for (; a + 3 * step < hi; a += 4 * step) {
      uint32_t u[4];
      bool in[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) u[k] = __ldg(col + a + k * step);
#pragma unroll
      for (int k = 0; k < 4; ++k) in[k] = (__ldg(front + (u[k] >> 5)) >> (u[k] & 31u)) & 1u;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (in[k]) {
          const uint32_t nd = __ldcg(srcdist + u[k]) + __ldg(w + a + k * step);
          b = nd < b ? nd : b;
          ++*hits;
        }
    }
    for (; a < hi; a += step) {
      const uint32_t u = __ldg(col + a);
      if ((__ldg(front + (u >> 5)) >> (u & 31u)) & 1u) {
        const uint32_t nd = __ldcg(srcdist + u) + __ldg(w + a);
        b = nd < b ? nd : b;
        ++*hits;
      }
    }
    return b;
  }
  __device__ __forceinline__ void improve(uint32_t v, uint32_t dv, uint32_t b) const {
    if (b < dv) {
      atomicMin(dist + v, b);
      atomicOr(changed + (v >> 5), 1u << (v & 31u));
    }
  }
};

__device__ __forceinline__ void add_counts(unsigned long long* c, unsigned long long scanned, unsigned long long hits) {
  for (int o = 16; o > 0; o >>= 1) {
    scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
    hits += __shfl_xor_sync(0xffffffffu, hits, o);
  }
  if ((threadIdx.x & 31u) == 0) {
    if (scanned) atomicAdd(c, scanned);
    if (hits) atomicAdd(c + 1, hits);
  }
}

// G lanes per row; the group's lanes share the row, so they take every branch together and the
// group minimum is a shuffle over the group's own lanes
template <int G>
__global__ void __launch_bounds__(256) k_pull_lanes(const uint32_t* __restrict__ rows, uint64_t count, PullRange R) {
  const uint32_t lane = threadIdx.x & 31u, lig = lane % G;
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane - lig));
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long scanned = 0, hits = 0;
  for (uint64_t base = warp * (32 / G); base < count; base += nwarps * (32 / G)) {
    const uint64_t i = base + lane / G;
    if (i >= count) continue;
    const uint32_t v = rows[i];
    const uint32_t dv = __ldcg(R.dist + v);
    if (dv < R.lo) continue;
    uint64_t a0, a1;
    R.range(v, &a0, &a1);
    if (a0 >= a1) continue;
    if (lig == 0) scanned += a1 - a0;
    uint32_t b = R.best(a0 + lig, a1, G, &hits);
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const uint32_t x = __shfl_xor_sync(gmask, b, o);
      b = x < b ? x : b;
    }
    if (lig == 0) R.improve(v, dv, b);
  }
  add_counts(R.counts, scanned, hits);
}

__device__ __forceinline__ uint32_t warp_min(uint32_t b) {
  for (int o = 16; o > 0; o >>= 1) {
    const uint32_t x = __shfl_xor_sync(0xffffffffu, b, o);
    b = x < b ? x : b;
  }
  return b;
}

// a CTA per row; each warp offers its own minimum (at most 8 atomics per improved row)
__global__ void __launch_bounds__(256) k_pull_cta(const uint32_t* __restrict__ rows, uint64_t count, PullRange R) {
  unsigned long long scanned = 0, hits = 0;
  for (uint64_t i = blockIdx.x; i < count; i += gridDim.x) {
    const uint32_t v = rows[i];
    const uint32_t dv = __ldcg(R.dist + v);
    if (dv < R.lo) continue;
    uint64_t a0, a1;
    R.range(v, &a0, &a1);
    if (a0 >= a1) continue;
    if (threadIdx.x == 0) scanned += a1 - a0;
    const uint32_t b = warp_min(R.best(a0 + threadIdx.x, a1, blockDim.x, &hits));
    if ((threadIdx.x & 31u) == 0) R.improve(v, dv, b);
  }
  add_counts(R.counts, scanned, hits);
}

// a CTA per 65536-arc chunk of the longest rows, cut to the light or heavy range
__global__ void __launch_bounds__(256) k_pull_chunks(const uint32_t* __restrict__ rows, const uint64_t* __restrict__ chunk_row,
                                                     const uint64_t* __restrict__ chunk_begin, uint64_t nchunks, uint64_t chunk,
                                                     PullRange R) {
  unsigned long long scanned = 0, hits = 0;
  for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const uint32_t v = rows[chunk_row[c]];
    const uint32_t dv = __ldcg(R.dist + v);
    if (dv < R.lo) continue;
    uint64_t a0, a1;
    R.range(v, &a0, &a1);
    const uint64_t c0 = chunk_begin[c], c1 = c0 + chunk;
    a0 = a0 > c0 ? a0 : c0;
    a1 = a1 < c1 ? a1 : c1;
    if (a0 >= a1) continue;
    if (threadIdx.x == 0) scanned += a1 - a0;
    const uint32_t b = warp_min(R.best(a0 + threadIdx.x, a1, blockDim.x, &hits));
    if ((threadIdx.x & 31u) == 0) R.improve(v, dv, b);
  }
  add_counts(R.counts, scanned, hits);
}

static int pull_binned(const DegreeBins& B, const PullRange& R, cudaStream_t s) {
  const uint32_t* r = B.rows;
  auto grid = [](uint64_t threads) { return grid_for(threads, 256, 8); };
  if (B.count[0]) k_pull_lanes<1><<<grid(B.count[0]), 256, 0, s>>>(r + B.start[0], B.count[0], R);
  if (B.count[1]) k_pull_lanes<2><<<grid(B.count[1] * 2), 256, 0, s>>>(r + B.start[1], B.count[1], R);
  if (B.count[2]) k_pull_lanes<4><<<grid(B.count[2] * 4), 256, 0, s>>>(r + B.start[2], B.count[2], R);
  if (B.count[3]) k_pull_lanes<8><<<grid(B.count[3] * 8), 256, 0, s>>>(r + B.start[3], B.count[3], R);
  if (B.count[4]) k_pull_lanes<16><<<grid(B.count[4] * 16), 256, 0, s>>>(r + B.start[4], B.count[4], R);
  if (B.count[5]) k_pull_lanes<32><<<grid(B.count[5] * 32), 256, 0, s>>>(r + B.start[5], B.count[5], R);
  if (B.count[6]) k_pull_cta<<<grid(B.count[6] * 256), 256, 0, s>>>(r + B.start[6], B.count[6], R);
  if (B.count[7])
    k_pull_chunks<<<grid(B.n_hub_chunks * 256), 256, 0, s>>>(r + B.start[7], B.hub_chunk_row, B.hub_chunk_begin, B.n_hub_chunks,
                                                            B.sched.hub_chunk, R);
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

// Which vertices have light arcs ([off, lend) non-empty) and which heavy ones ([lend, off+1)):
// one bit each, so that the passes below test a word instead of reading three offsets per vertex.
__global__ void k_sssp_classes(uint64_t n, const uint64_t* __restrict__ off, const uint64_t* __restrict__ lend,
                               uint32_t* __restrict__ lbits, uint32_t* __restrict__ hbits) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < n; base += stride) {
    const uint64_t v = base + (threadIdx.x & 31u);
    bool light = false, heavy = false;
    if (v < n) {
      const uint64_t a0 = off[v], am = lend[v], a1 = off[v + 1];
      light = am > a0;
      heavy = a1 > am;
    }
    const uint32_t lw = __ballot_sync(0xffffffffu, light), hw = __ballot_sync(0xffffffffu, heavy);
    if ((threadIdx.x & 31u) == 0) {
      lbits[base >> 5] = lw;
      hbits[base >> 5] = hw;
    }
  }
}

int sssp_relax_binned_offer(cudaStream_t stream, const DegreeBins& B, const uint32_t* front, const uint64_t* off,
                            const uint64_t* lend, bool heavy, const uint32_t* col, const uint32_t* w, const uint32_t* srcdist,
                            uint32_t* offers, uint32_t* touched, const uint32_t* known, const OwnHeads& own,
                            unsigned long long* arcs) {
  RelaxRange R{front, off, lend, col, w, offers, touched, arcs, heavy, srcdist, known, own};
  return relax_binned<true>(B, R, stream);
}

int sssp_pull_binned(cudaStream_t stream, const DegreeBins& B, const uint32_t* front, const uint64_t* off, const uint64_t* lend,
                     bool heavy, const uint32_t* col, const uint32_t* w, const uint32_t* srcdist, uint32_t* dist, uint32_t* changed,
                     uint32_t lo, unsigned long long* counts) {
  PullRange P{front, off, lend, col, w, dist, changed, counts, heavy, lo, srcdist};
  return pull_binned(B, P, stream);
}

int sssp_split_rows(cudaStream_t stream, uint64_t rows, const uint64_t* off, const uint32_t* col, const uint32_t* w, uint32_t delta,
                    uint32_t* ocol, uint32_t* ow, uint64_t* lend) {
  if (rows) k_split_light_heavy<<<grid_for(rows * 32, 256), 256, 0, stream>>>(rows, off, col, w, delta, ocol, ow, lend);
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

constexpr int kStage = 512;  // items per list that a warp stages in shared memory (2 lists x 8 warps: 32 KB)

// Classify the vertices improved by a pass (bits of `changed`, one lane per word, cleared here):
// below the limit a vertex with light arcs joins the near queue and one with heavy arcs the
// bucket list (once: `inbucket`), and leaves the far set; at or above the limit it joins the far
// set (a bitmap, `infar`).  Vertices without out-arcs are dropped.  counters[0] and [4] are the
// queue and list lengths, counters[2] the far set's size.
__global__ void __launch_bounds__(256) k_sssp_classify(uint64_t nwords, uint32_t* __restrict__ changed, const uint32_t* __restrict__ dist,
                                const uint32_t* __restrict__ lbits, const uint32_t* __restrict__ hbits, uint32_t near_limit,
                                uint32_t* __restrict__ near, uint32_t* __restrict__ infar,
                                uint32_t* __restrict__ inbucket, uint32_t* __restrict__ blist, uint32_t* __restrict__ counters) {
  __shared__ uint32_t stage[8][2 * kStage];
  WarpLists<2, kStage> out(stage[threadIdx.x >> 5]);
  int far_delta = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < nwords; base += stride) {
    const uint64_t wi = base + (threadIdx.x & 31u);
    uint32_t bits = 0, fbits = 0, bbits = 0, lw = 0, hw = 0;
    if (wi < nwords) {
      bits = changed[wi];
      if (bits) {
        changed[wi] = 0;
        fbits = infar[wi];
        bbits = inbucket[wi];
        lw = lbits[wi];
        hw = hbits[wi];
      }
    }
    uint32_t set_far = 0, clear_far = 0, set_bucket = 0;
    while (__any_sync(0xffffffffu, bits != 0)) {
      bool to_near = false, to_bucket = false;
      uint32_t v = 0;
      if (bits) {
        const uint32_t b = __ffs(bits) - 1;
        bits &= bits - 1;
        v = (uint32_t)(wi << 5) + b;
        const bool light = (lw >> b) & 1u, heavy = (hw >> b) & 1u;
        if (light || heavy) {
          if (dist[v] < near_limit) {
            to_near = light;
            if (heavy && !(bbits & (1u << b))) {
              to_bucket = true;
              set_bucket |= 1u << b;
            }
            if (fbits & (1u << b)) clear_far |= 1u << b;
          } else if (!(fbits & (1u << b))) {
            set_far |= 1u << b;
          }
        }
      }
      out.push<0>(to_near, v, counters, near);
      out.push<1>(to_bucket, v, counters + 4, blist);
    }
    if (set_far | clear_far) infar[wi] = (fbits | set_far) & ~clear_far;  // one lane owns the word
    if (set_bucket) inbucket[wi] = bbits | set_bucket;
    far_delta += __popc(set_far) - __popc(clear_far);
  }
  out.flush<0>(counters, near);
  out.flush<1>(counters + 4, blist);
  far_delta = __reduce_add_sync(0xffffffffu, far_delta);
  if ((threadIdx.x & 31u) == 0 && far_delta) atomicAdd(counters + 2, (uint32_t)far_delta);
}

// The bucket's heavy arcs have been relaxed: its members leave the bucket list.
__global__ void k_bucket_clear(const uint32_t* __restrict__ blist, uint64_t nb, uint32_t* __restrict__ inbucket) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nb; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = blist[i];
    atomicAnd(inbucket + (v >> 5), ~(1u << (v & 31u)));
  }
}

// The source joins the near queue (light arcs) and the bucket list (heavy arcs).
__global__ void k_sssp_seed(uint32_t src, const uint64_t* __restrict__ off, const uint64_t* __restrict__ lend,
                            uint32_t* __restrict__ dist, uint32_t* __restrict__ near, uint32_t* __restrict__ inbucket,
                            uint32_t* __restrict__ blist, uint32_t* __restrict__ counters) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  dist[src] = 0;
  if (lend[src] > off[src]) near[counters[0]++] = src;
  if (off[src + 1] > lend[src]) {
    blist[counters[4]++] = src;
    inbucket[src >> 5] |= 1u << (src & 31u);
  }
}

// Near-far split when the limit rises: every vertex of the far set (bitmap `infar`) whose
// distance is now below the limit leaves it for the near queue (light arcs) and the bucket list
// (heavy arcs; once: `inbucket`), as in k_sssp_classify; the others stay.  counters[2] (the far
// set's size) drops by the vertices that left, counters[3] gets the smallest distance left.  A
// scan of the bitmap reads the distances of far vertices in vertex order, 32 to a word.
__global__ void __launch_bounds__(256) k_far_split(uint64_t nwords, uint32_t* __restrict__ infar, const uint32_t* __restrict__ dist,
                                                   uint32_t near_limit, const uint32_t* __restrict__ lbits,
                                                   const uint32_t* __restrict__ hbits, uint32_t* __restrict__ near,
                                                   uint32_t* __restrict__ inbucket, uint32_t* __restrict__ blist,
                                                   uint32_t* __restrict__ counters) {
  __shared__ uint32_t stage[8][2 * kStage];
  WarpLists<2, kStage> out(stage[threadIdx.x >> 5]);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t dmin = 0xffffffffu, nmoved = 0;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < nwords; base += stride) {
    const uint64_t wi = base + (threadIdx.x & 31u);
    uint32_t bits = wi < nwords ? infar[wi] : 0u;
    const uint32_t fbits = bits;
    uint32_t moved = 0, set_bucket = 0, bbits = 0, lw = 0, hw = 0;
    if (bits) {
      bbits = inbucket[wi];
      lw = lbits[wi];
      hw = hbits[wi];
    }
    while (__any_sync(0xffffffffu, bits != 0)) {
      bool to_near = false, to_bucket = false;
      uint32_t v = 0;
      if (bits) {
        const uint32_t b = __ffs(bits) - 1;
        bits &= bits - 1;
        v = (uint32_t)(wi << 5) + b;
        const uint32_t d = dist[v];
        if (d < near_limit) {
          moved |= 1u << b;
          to_near = (lw >> b) & 1u;
          if (((hw >> b) & 1u) && !(bbits & (1u << b))) {
            to_bucket = true;
            set_bucket |= 1u << b;
          }
        } else {
          dmin = min(dmin, d);
        }
      }
      out.push<0>(to_near, v, counters, near);
      out.push<1>(to_bucket, v, counters + 4, blist);
    }
    if (moved) infar[wi] = fbits & ~moved;
    if (set_bucket) inbucket[wi] = bbits | set_bucket;
    nmoved += __popc(moved);
  }
  out.flush<0>(counters, near);
  out.flush<1>(counters + 4, blist);
  dmin = __reduce_min_sync(0xffffffffu, dmin);
  nmoved = __reduce_add_sync(0xffffffffu, nmoved);
  if ((threadIdx.x & 31u) == 0) {
    if (dmin != 0xffffffffu) atomicMin(counters + 3, dmin);
    if (nmoved) atomicSub(counters + 2, nmoved);
  }
}

struct AddU64 {
  __device__ __forceinline__ uint64_t operator()(uint64_t a, uint64_t b) const { return a + b; }
};

// Bucket width of the near-far split.  Default: 3/8 of the mean arc weight (RMAT-26, weights in
// [1, 255], heavy passes pulled: delta 24 / 32 / 40 / 48 / 64 / 96 / 128 gave 23.3 / 20.6 / 20.4
// / 19.9 / 20.4 / 22.2 / 25.0 ms); 0 relaxes every improved vertex at once (Bellman-Ford frontier).
// The GRE_SSSP_DELTA environment variable overrides it.
int sssp_delta(gre_graph g, uint32_t* delta) {
  if (const char* e = getenv("GRE_SSSP_DELTA")) {
    *delta = (uint32_t)strtoul(e, nullptr, 10);
    return GRE_SUCCESS;
  }
  if (g->w32_mean < 0) {
    uint64_t* dsum = nullptr;
    GRE_CHECK(ws_array(g, WS_COUNTERS, 1, &dsum));
    size_t tb = 0;
    cub::DeviceReduce::Reduce(nullptr, tb, g->w32, dsum, g->m, AddU64(), (uint64_t)0, g->stream);
    void* tmp = nullptr;
    GRE_CHECK(g->ws.get(WS_CUB, tb, &tmp));
    GRE_CUDA(cub::DeviceReduce::Reduce(tmp, tb, g->w32, dsum, g->m, AddU64(), (uint64_t)0, g->stream));
    uint64_t sum = 0;
    GRE_CUDA(cudaMemcpyAsync(&sum, dsum, sizeof sum, cudaMemcpyDeviceToHost, g->stream));
    GRE_CUDA(cudaStreamSynchronize(g->stream));
    g->w32_mean = g->m ? (double)sum / (double)g->m : 1.0;
  }
  const double d = g->w32_mean * 0.375;
  *delta = d < 1.0 ? 1u : d > 1e9 ? 1000000000u : (uint32_t)d;
  return GRE_SUCCESS;
}

// counters: [0] near appends, [1] overflow flag, [2] size of the far set, [3] smallest far
// distance left by a split, [4] bucket-list appends (from its size)
static int init_counters(gre_graph g, uint32_t* cnt, uint32_t near, uint32_t nfar, uint32_t nbucket) {
  const uint32_t h[8] = {near, 0, nfar, 0xffffffffu, nbucket, 0, 0, 0};  // pageable: staged before the call returns
  GRE_CUDA(cudaMemcpyAsync(cnt, h, sizeof h, cudaMemcpyHostToDevice, g->stream));
  return GRE_SUCCESS;
}

// Resident CTAs of the relaxation kernel per SM: the grid is exactly one wave, so that no
// CTA starts its tiles late.
template <bool OFFER>
static int relax_blocks_per_sm() {
  static int per_sm = 0;
  if (!per_sm) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sssp_relax<OFFER>, kTileThreads, 0) != cudaSuccess || b < 1) b = 1;
    per_sm = b;
  }
  return per_sm;
}

uint64_t sssp_tile_arcs() { return kTile; }

// Frontiers of at least n / binned_frontier() vertices are relaxed through the degree bins
// (default 16; the GRE_SSSP_BINNED environment variable overrides it, 0 = never).
static uint64_t binned_frontier() {
  if (const char* e = getenv("GRE_SSSP_BINNED")) return strtoull(e, nullptr, 10);
  return 16;
}
uint64_t sssp_binned_divisor() { return binned_frontier(); }

// Whether the large heavy passes pull (over the vertices that can still improve) instead of
// pushing (along the bucket's heavy arcs), where the weights allow it (g->w32_symmetric).
// Default on; the GRE_SSSP_PULL environment variable set to 0 keeps the push form.
static bool pull_enabled() {
  if (const char* e = getenv("GRE_SSSP_PULL")) return strtoul(e, nullptr, 10) != 0;
  return true;
}
bool sssp_pull_enabled() { return pull_enabled(); }

// A heavy pass whose bucket has at least m / d heavy arcs pulls even when the bucket has fewer
// than n / sssp_binned_divisor() members (a few hubs can carry a large share of the arcs): d from
// GRE_SSSP_PULL_ARCS, default 16; 0 decides by the member count alone.
static uint64_t pull_arcs_divisor() {
  if (const char* e = getenv("GRE_SSSP_PULL_ARCS")) return strtoull(e, nullptr, 10);
  return 16;
}
uint64_t sssp_pull_arcs_divisor() { return pull_arcs_divisor(); }

// The tuner picks the row schedule for the PageRank gather (RMAT-26: 16 arcs per lane, a warp up
// to 65536 arcs); SSSP's pushes wait on two dependent loads per four arcs, so longer chains per
// lane cost them (RMAT-26 SSSP 18.0 -> 19.4 ms under that schedule).  Their bins keep at most 8
// arcs per lane and a CTA from 16384 arcs.
int sssp_bins(gre_graph g, bool in, const DegreeBins** out) {
  GRE_CHECK(ensure_bins(g, in));
  const DegreeBins& B = in ? g->bins_in : g->bins_out;
  if (B.sched.lane_arcs <= 8 && B.sched.cta_min <= 16384) {
    *out = &B;
    return GRE_SUCCESS;
  }
  RowSchedule s = B.sched;
  s.lane_arcs = std::min<uint32_t>(s.lane_arcs, 8);
  s.cta_min = std::min<uint64_t>(s.cta_min, 16384);
  s.hub_chunk = 65536;
  s.seg_window = 0;
  DegreeBins& S = g->bins_sssp;
  if (!S.ready || S.sched.lane_arcs != s.lane_arcs || S.sched.cta_min != s.cta_min || S.sched.hub_chunk != s.hub_chunk)
    GRE_CHECK(build_bins(g, S, in ? g->roff : g->off, in ? g->rcol : g->col, s));
  *out = &S;
  return GRE_SUCCESS;
}

// The relaxation of one frontier pass: tile starts, then k_sssp_relax over one wave of CTAs.
int sssp_relax_tiles(cudaStream_t stream, const uint32_t* queue, uint64_t nq, const uint64_t* prefix, uint64_t total,
                     uint32_t* tstart, const uint64_t* base, const uint32_t* col, const uint32_t* w, const uint32_t* srcdist,
                     uint32_t* dist, uint32_t* changed, uint32_t* error, const uint32_t* known, const OwnHeads& own) {
  if (!total) return GRE_SUCCESS;
  const uint64_t ntiles = (total + kTile - 1) / kTile;
  k_tile_starts<<<grid_for(nq, 256), 256, 0, stream>>>(prefix, nq, tstart);
  // the arc count is a launch argument: read inside the kernel instead, the relaxation
  // measured 1.7x slower on RMAT-26
  const bool offer = srcdist != dist;
  const int grid = (int)std::min<uint64_t>(ntiles, (uint64_t)num_sms() * (offer ? relax_blocks_per_sm<true>() : relax_blocks_per_sm<false>()));
  if (!offer)
    k_sssp_relax<false><<<grid, kTileThreads, 0, stream>>>(queue, nq, prefix, total, tstart, base, col, w, nullptr, dist, changed,
                                                           error, nullptr, OwnHeads());
  else
    k_sssp_relax<true><<<grid, kTileThreads, 0, stream>>>(queue, nq, prefix, total, tstart, base, col, w, srcdist, dist, changed,
                                                          error, known, own);
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

// Light/heavy split of the arcs for bucket width delta (built once per graph, weights and delta).
static int ensure_split(gre_graph g, uint32_t delta) {
  auto& sp = g->sssp_split;
  if (sp.lsplit && sp.delta == delta) return GRE_SUCCESS;
  sp.release();
  const uint64_t n = g->n, m = g->m;
  cudaError_t e = cudaMalloc(&sp.col, sizeof(uint32_t) * (m ? m : 1));
  if (e == cudaSuccess) e = cudaMalloc(&sp.w, sizeof(uint32_t) * (m ? m : 1));
  if (e == cudaSuccess) e = cudaMalloc(&sp.lsplit, sizeof(uint64_t) * (n ? n : 1));
  if (e != cudaSuccess) {
    sp.release();
    return cuda_status(e, "cudaMalloc (SSSP light/heavy split)", __FILE__, __LINE__);
  }
  k_split_light_heavy<<<grid_for(n * 32, 256), 256, 0, g->stream>>>(n, g->off, g->col, g->w32, delta, sp.col, sp.w, sp.lsplit);
  GRE_LAUNCH_CHECK();
  sp.delta = delta;
  return GRE_SUCCESS;
}

// One SSSP.  With delta > 0, near-far buckets of width delta with the light/heavy split of
// delta-stepping (Meyer and Sanders 2003): inside a bucket only light arcs (w < delta) are
// relaxed, repeatedly, as the bucket's distances settle; when the bucket is done, the heavy arcs
// of every vertex it settled are relaxed once (they can only reach later buckets).  delta = 0:
// Bellman-Ford frontier over all arcs.
static int sssp_one(gre_graph g, uint32_t src, uint32_t* dist, gre_stats* st, bool record, uint32_t delta) {
  const uint64_t n = g->n;
  const uint64_t nwords = (n + 31) >> 5;
  if (delta) GRE_CHECK(ensure_split(g, delta));
  const uint64_t* off = g->off;
  const uint64_t* lend = delta ? g->sssp_split.lsplit : g->off + 1;  // end of each row's light arcs
  const uint32_t* col = delta ? g->sssp_split.col : g->col;
  const uint32_t* w = delta ? g->sssp_split.w : g->w32;
  uint32_t *qa, *qb, *changed, *cnt, *infar, *tstart, *inbucket, *blist;
  uint64_t *deg, *prefix;
  GRE_CHECK(ws_array(g, WS_A, n, &qa));
  GRE_CHECK(ws_array(g, WS_B, n, &qb));
  GRE_CHECK(ws_array(g, WS_C, nwords, &changed));
  GRE_CHECK(ws_array(g, WS_F, n + 1, &deg));
  GRE_CHECK(ws_array(g, WS_G, n + 1, &prefix));
  GRE_CHECK(ws_array(g, WS_I, g->m / kTile + 2, &tstart));
  GRE_CHECK(ws_array(g, WS_J, nwords, &infar));
  GRE_CHECK(ws_array(g, WS_K, nwords, &inbucket));
  GRE_CHECK(ws_array(g, WS_L, n, &blist));
  uint32_t *lbits, *hbits;
  GRE_CHECK(ws_array(g, WS_SSSP_L, nwords, &lbits));
  GRE_CHECK(ws_array(g, WS_SSSP_H, nwords, &hbits));
  // 8 uint32 counters, then the binned passes' arc count and the pull passes' scanned arcs and hits
  GRE_CHECK(ws_array(g, WS_COUNTERS, 14, &cnt));
  unsigned long long* binned_arcs = (unsigned long long*)(cnt + 8);
  unsigned long long* pull_counts = (unsigned long long*)(cnt + 10);
  const bool pull = g->w32_symmetric && pull_enabled();
  // large frontiers go through the degree bins of the CSR (the symmetric CSC is the CSR)
  const bool sym = g->symmetric();
  const DegreeBins* pbins = nullptr;
  GRE_CHECK(sssp_bins(g, sym, &pbins));
  const DegreeBins& bins = *pbins;
  const uint64_t bdiv = binned_frontier();
  const uint64_t pdiv = pull_arcs_divisor();
  size_t cubbytes = 0;
  void* cubtmp = nullptr;
  cub::DeviceScan::ExclusiveSum(nullptr, cubbytes, deg, prefix, n + 1, g->stream);
  GRE_CHECK(g->ws.get(WS_CUB, cubbytes, &cubtmp));
  GRE_CUDA(cudaMemsetAsync(dist, 0xff, sizeof(uint32_t) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(changed, 0, sizeof(uint32_t) * nwords, g->stream));
  GRE_CUDA(cudaMemsetAsync(infar, 0, sizeof(uint32_t) * nwords, g->stream));
  GRE_CUDA(cudaMemsetAsync(inbucket, 0, sizeof(uint32_t) * nwords, g->stream));
  GRE_CUDA(cudaMemsetAsync(binned_arcs, 0, 3 * sizeof(unsigned long long), g->stream));
  k_sssp_classes<<<grid_for(n, 256, 8), 256, 0, g->stream>>>(n, off, lend, lbits, hbits);
  uint32_t limit = delta ? delta : 0xffffffffu;
  uint64_t nq = 0, nfar = 0, nb = 0, relaxed = 0, bytes = 0;
  uint32_t* q = qa;
  uint32_t* nqueue = qb;
  uint32_t steps = 0;
  uint32_t h[8];
  auto read_counters = [&]() -> int {
    GRE_CUDA(cudaMemcpyAsync(h, cnt, sizeof h, cudaMemcpyDeviceToHost, g->stream));
    GRE_CUDA(cudaStreamSynchronize(g->stream));
    if (h[1]) {
      set_error("gre_sssp: frontier tile overflow");
      return GRE_FAILURE;
    }
    return GRE_SUCCESS;
  };
  GRE_CHECK(init_counters(g, cnt, 0, 0, 0));
  k_sssp_seed<<<1, 32, 0, g->stream>>>(src, off, lend, dist, q, inbucket, blist, cnt);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(read_counters());
  nq = h[0];
  nb = h[4];
  // one relaxation pass over `list` (light or heavy ranges), the improvements classified into
  // the next near queue, the bucket list and the far set
  auto pass = [&](const uint32_t* list, uint64_t nlist, bool heavy, uint32_t* out_near) -> int {
    bool bins_form = bdiv && nlist >= n / bdiv && nlist > 0;
    uint64_t total = 0;
    if (!bins_form) {  // the arcs of the frontier, for the tiles
      if (heavy) k_sssp_degrees<true><<<grid_for(nlist, 256), 256, 0, g->stream>>>(list, nlist, off, lend, deg);
      else k_sssp_degrees<false><<<grid_for(nlist, 256), 256, 0, g->stream>>>(list, nlist, off, lend, deg);
      GRE_CUDA(cub::DeviceScan::ExclusiveSum(cubtmp, cubbytes, deg, prefix, nlist + 1, g->stream));
      GRE_CUDA(cudaMemcpyAsync(&total, prefix + nlist, sizeof total, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      // a small bucket with many heavy arcs (hubs among its members) pulls them instead
      if (heavy && pull && bdiv && pdiv && total && total * pdiv >= g->m) bins_form = true;
    }
    if (bins_form) {
      // the heavy pass's frontier is the bucket, already a bitmap; a light frontier is made one
      // in the scan buffer (free in this form of the pass)
      uint32_t* front = inbucket;
      if (!heavy) {
        front = (uint32_t*)deg;
        GRE_CUDA(cudaMemsetAsync(front, 0, sizeof(uint32_t) * nwords, g->stream));
        k_queue_to_bits<<<grid_for(nlist, 256), 256, 0, g->stream>>>(list, nlist, front);
      }
      GRE_CHECK(init_counters(g, cnt, 0, (uint32_t)nfar, (uint32_t)nb));
      if (pull && heavy) {
        // the bucket's heavy arcs: only vertices at or above the limit can improve (heavy arcs
        // from the bucket land there).  (Light passes push: every unsettled vertex would have to
        // scan its light arcs at every pass of the bucket, measured slower than the push.)
        PullRange P{front, off, lend, col, w, dist, changed, pull_counts, true, limit, dist};
        GRE_CHECK(pull_binned(bins, P, g->stream));
        bytes += 16 * n;  // per row: its id, distance and range bounds (arcs at the end)
      } else {
        RelaxRange R{front, off, lend, col, w, dist, changed, binned_arcs, heavy, nullptr};
        GRE_CHECK(relax_binned<false>(bins, R, g->stream));
      }
      k_sssp_classify<<<grid_for(nwords, 256, 4), 256, 0, g->stream>>>(nwords, changed, dist, lbits, hbits, limit, out_near, infar,
                                                                        inbucket, blist, cnt);
      GRE_LAUNCH_CHECK();
      GRE_CHECK(read_counters());
      bytes += 4 * n + n / 8 + 8 * (uint64_t)(h[0] + h[2] - nfar + h[4] - nb);  // rows scanned, bitmap (arcs below)
      nfar = h[2];
      nb = h[4];
      ++steps;
      return GRE_SUCCESS;
    }
    GRE_CHECK(init_counters(g, cnt, 0, (uint32_t)nfar, (uint32_t)nb));
    if (total) {
      GRE_CHECK(sssp_relax_tiles(g->stream, list, nlist, prefix, total, tstart, heavy ? lend : off, col, w, dist, dist, changed,
                                 cnt + 1, nullptr, OwnHeads()));
      k_sssp_classify<<<grid_for(nwords, 256, 4), 256, 0, g->stream>>>(nwords, changed, dist, lbits, hbits, limit, out_near, infar,
                                                                        inbucket, blist, cnt);
    }
    GRE_LAUNCH_CHECK();
    GRE_CHECK(read_counters());
    relaxed += total;
    bytes += 16 * nlist + 12 * total + 8 * (uint64_t)(h[0] + h[2] - nfar + h[4] - nb);
    nfar = h[2];
    nb = h[4];
    ++steps;
    return GRE_SUCCESS;
  };
  for (;;) {
    while (nq > 0) {  // light supersteps of the bucket
      GRE_CHECK(pass(q, nq, false, nqueue));
      nq = h[0];
      std::swap(q, nqueue);
      if (record) stats_record(st, nq);
    }
    if (nb > 0) {  // the bucket is settled: its heavy arcs, once
      // heavy arcs land at or above the limit, so the pass normally appends nothing below it;
      // anything it does append (a distance that wrapped around 2^32) goes after the members
      const uint64_t members = nb;
      GRE_CHECK(pass(blist, members, true, q));
      k_bucket_clear<<<grid_for(members, 256), 256, 0, g->stream>>>(blist, members, inbucket);
      GRE_LAUNCH_CHECK();
      if (nb > members) {  // move them to the front through scratch (the ranges may overlap)
        const size_t bytes_extra = sizeof(uint32_t) * (nb - members);
        GRE_CUDA(cudaMemcpyAsync(deg, blist + members, bytes_extra, cudaMemcpyDeviceToDevice, g->stream));
        GRE_CUDA(cudaMemcpyAsync(blist, deg, bytes_extra, cudaMemcpyDeviceToDevice, g->stream));
      }
      nb -= members;
      nq = h[0];
      if (record) stats_record(st, nq);
      if (nq > 0 || nb > 0) continue;
    }
    if (nfar == 0) break;
    // the near queue is empty: raise the limit (past empty buckets) and pull the far vertices below it
    uint32_t lowest = 0;
    for (int p = 0; nq == 0 && nb == 0 && nfar > 0; ++p) {
      if (p == 2) {  // the second pass starts at the smallest distance left: cannot come back empty
        set_error("gre_sssp: near-far split made no progress");
        return GRE_FAILURE;
      }
      if (p == 0) limit = limit > 0xffffffffu - delta ? 0xffffffffu : limit + delta;
      else limit = lowest > 0xffffffffu - delta ? 0xffffffffu : lowest + delta;
      GRE_CHECK(init_counters(g, cnt, 0, (uint32_t)nfar, 0));
      k_far_split<<<grid_for(nwords, 256, 4), 256, 0, g->stream>>>(nwords, infar, dist, limit, lbits, hbits, q, inbucket, blist,
                                                                    cnt);
      GRE_LAUNCH_CHECK();
      GRE_CHECK(read_counters());
      bytes += 4 * nwords + 4 * nfar + 4 * (uint64_t)(h[0] + h[4]);
      nq = h[0];
      nfar = h[2];
      nb = h[4];
      lowest = h[3];
    }
  }
  unsigned long long bc[3] = {0, 0, 0};
  GRE_CUDA(cudaMemcpyAsync(bc, binned_arcs, sizeof bc, cudaMemcpyDeviceToHost, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  relaxed += bc[0] + bc[1];
  bytes += 12 * bc[0];              // push: column + weight + distance probe per arc
  bytes += 4 * bc[1] + 8 * bc[2];   // pull: column per arc scanned (+ L2-held bitmap), weight + distance per hit
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
  uint32_t delta = 0;
  GRE_CHECK(sssp_delta(g, &delta));  // before any workspace pointer is taken (it may grow WS_CUB)
  uint32_t *dfinal, *dd;
  int32_t* lv;
  GRE_CHECK(prepare_output(g, dist, (uint64_t)nsrc * n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, nsrc, 4, (void**)&dd));
  GRE_CHECK(ws_array(g, WS_H, n, &lv));
  RunTimer timer(g);
  uint64_t edges = 0;
  for (uint32_t i = 0; i < nsrc; ++i) {
    GRE_CHECK(sssp_one(g, hs[i], dd + (uint64_t)i * n, st, nsrc == 1, delta));
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
