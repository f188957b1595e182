// Top-down (push) step of the 64-sources-per-word BFS, used when the frontier is sparse.
//
// The bottom-up step (every vertex ORs the frontier words of its in-neighbours) reads every arc
// of every not-fully-visited vertex each level; with a small frontier that is almost all wasted.
// The push step visits only the arcs of frontier vertices: acc[v] |= F_d[u] & ~seen[v] with
// 64-bit atomicOr, then one pass over the vertices commits acc into the next frontier word and
// the seen word.  OR is order-independent, so both directions give the same frontier words.
#pragma once
#include "gre_internal.cuh"

namespace gre {
namespace ms {

// Vertices whose frontier word is non-zero, and the sum of their out-degrees.
static __global__ void k_frontier_list(uint64_t n, const unsigned long long* __restrict__ f, const uint64_t* __restrict__ off,
                                       uint32_t* __restrict__ list, unsigned int* __restrict__ count,
                                       unsigned long long* __restrict__ arcs) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long deg = 0;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < n; base += stride) {
    const uint64_t v = base + (threadIdx.x & 31u);
    const bool nz = v < n && f[v] != 0ull;
    const uint32_t pos = warp_append(count, nz);
    if (nz) {
      list[pos] = (uint32_t)v;
      deg += off[v + 1] - off[v];
    }
  }
  for (int o = 16; o > 0; o >>= 1) deg += __shfl_xor_sync(0xffffffffu, deg, o);
  if ((threadIdx.x & 31u) == 0 && deg) atomicAdd(arcs, deg);
}

// Warp per frontier vertex, lanes over its out-arcs.
static __global__ void __launch_bounds__(256) k_push(const uint32_t* __restrict__ list, const unsigned int* __restrict__ count,
                                                     const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                     const unsigned long long* __restrict__ fd, const unsigned long long* __restrict__ seen,
                                                     unsigned long long* __restrict__ acc) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t cnt = *count;
  for (uint64_t i = warp; i < cnt; i += nwarps) {
    const uint32_t u = list[i];
    const unsigned long long fu = fd[u];
    const uint64_t a1 = off[u + 1];
    for (uint64_t a = off[u] + lane; a < a1; a += 32) {
      const uint32_t v = __ldg(col + a);
      const unsigned long long bits = fu & ~seen[v];
      if (bits && (acc[v] & bits) != bits) atomicOr(acc + v, bits);
    }
  }
}

// Bottom-up (pull) step over the degree bins of the in-arcs: acc[v] = (OR over in-neighbours u
// of F_d[u]) & ~seen[v].  Rows of up to 64 arcs use groups of L lanes (a thread per row stops
// as soon as every unseen source is found); longer rows use a warp per row that stops, for the
// whole warp at once, when the OR of its lanes covers every unseen source.  A vertex whose
// sources are all seen is skipped.  Work per row is therefore bounded by its own degree: no
// thread walks a hub's arcs alone.
template <int L>
static __global__ void __launch_bounds__(256) k_pull_small(const uint32_t* __restrict__ rows, uint64_t count,
                                                           unsigned long long full, const uint64_t* __restrict__ roff,
                                                           const uint32_t* __restrict__ rcol, const unsigned long long* __restrict__ fd,
                                                           const unsigned long long* __restrict__ seen, unsigned long long* __restrict__ acc,
                                                           unsigned long long* __restrict__ scanned_out) {
  constexpr int G = 32 / L;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lig = lane % L;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long scanned = 0;
  for (uint64_t base = warp * G; base < count; base += nwarps * G) {
    const uint64_t i = base + lane / L;
    unsigned long long got = 0, want = 0;
    uint32_t v = 0;
    if (i < count) {
      v = rows[i];
      want = full & ~seen[v];
      if (want) {
        const uint64_t a1 = roff[v + 1];
        for (uint64_t a = roff[v] + lig; a < a1; a += L) {
          got |= fd[__ldg(rcol + a)];
          ++scanned;
          if (L == 1 && (got & want) == want) break;
        }
      }
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) got |= __shfl_xor_sync(0xffffffffu, got, o);
    if (i < count && lig == 0 && (got & want)) acc[v] = got & want;
  }
  for (int o = 16; o > 0; o >>= 1) scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
  if (lane == 0 && scanned) atomicAdd(scanned_out, scanned);
}

static __global__ void __launch_bounds__(256) k_pull_warp(const uint32_t* __restrict__ rows, uint64_t count, unsigned long long full,
                                                          const uint64_t* __restrict__ roff, const uint32_t* __restrict__ rcol,
                                                          const unsigned long long* __restrict__ fd,
                                                          const unsigned long long* __restrict__ seen, unsigned long long* __restrict__ acc,
                                                          unsigned long long* __restrict__ scanned_out) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long scanned = 0;
  for (uint64_t i = warp; i < count; i += nwarps) {
    const uint32_t v = rows[i];
    const unsigned long long want = full & ~seen[v];
    if (!want) continue;  // uniform: one row per warp
    unsigned long long got = 0;
    const uint64_t a0 = roff[v], a1 = roff[v + 1];
    for (uint64_t b = a0; b < a1; b += 32) {
      if (b + lane < a1) {
        got |= fd[__ldg(rcol + b + lane)];
        ++scanned;
      }
      const unsigned int lo = __reduce_or_sync(0xffffffffu, (unsigned int)(got & 0xffffffffull));
      const unsigned int hi = __reduce_or_sync(0xffffffffu, (unsigned int)(got >> 32));
      got = ((unsigned long long)hi << 32) | lo;
      if ((got & want) == want) break;  // the same decision in every lane
    }
    if (lane == 0 && (got & want)) acc[v] = got & want;
  }
  for (int o = 16; o > 0; o >>= 1) scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
  if (lane == 0 && scanned) atomicAdd(scanned_out, scanned);
}

// Launch the pull over every row with in-arcs (bins of the CSC).
static inline int pull(const DegreeBins& B, unsigned long long full, const uint64_t* roff, const uint32_t* rcol,
                       const unsigned long long* fd, const unsigned long long* seen, unsigned long long* acc,
                       unsigned long long* scanned, cudaStream_t s) {
  const uint32_t* r = B.rows;
  auto grid = [](uint64_t threads) { return grid_for(threads, 256, 8); };
  if (B.count[0]) k_pull_small<1><<<grid(B.count[0]), 256, 0, s>>>(r + B.start[0], B.count[0], full, roff, rcol, fd, seen, acc, scanned);
  if (B.count[1]) k_pull_small<2><<<grid(B.count[1] * 2), 256, 0, s>>>(r + B.start[1], B.count[1], full, roff, rcol, fd, seen, acc, scanned);
  if (B.count[2]) k_pull_small<4><<<grid(B.count[2] * 4), 256, 0, s>>>(r + B.start[2], B.count[2], full, roff, rcol, fd, seen, acc, scanned);
  if (B.count[3]) k_pull_small<8><<<grid(B.count[3] * 8), 256, 0, s>>>(r + B.start[3], B.count[3], full, roff, rcol, fd, seen, acc, scanned);
  if (B.count[4]) k_pull_small<16><<<grid(B.count[4] * 16), 256, 0, s>>>(r + B.start[4], B.count[4], full, roff, rcol, fd, seen, acc, scanned);
  const uint64_t nlong = B.count[5] + B.count[6] + B.count[7];  // contiguous in the bin list
  if (nlong) k_pull_warp<<<grid(nlong * 32), 256, 0, s>>>(r + B.start[5], nlong, full, roff, rcol, fd, seen, acc, scanned);
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

// fnext[v] = acc[v]; seen[v] |= acc[v]; acc[v] = 0.  When `levels` is given (k sources, rows of
// n int32), writes next_level for every new (source, vertex) pair, one bit at a time across the
// warp so that the writes of one source coalesce.  counters[0] += vertices with new bits,
// counters[1] += new (source, vertex) pairs, *live |= every new bit: the sources whose next
// frontier is not empty.  Only those can reach a vertex at the next level, so the pull stops
// looking for the others (a source in a small component would otherwise keep every vertex of
// the large one scanning all its arcs at every level).
static __global__ void k_commit(uint64_t n, unsigned long long* __restrict__ acc, unsigned long long* __restrict__ seen,
                                unsigned long long* __restrict__ fnext, int32_t* __restrict__ levels, int32_t next_level,
                                unsigned long long* __restrict__ counters, unsigned long long* __restrict__ live) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long found_v = 0, found_bits = 0, any_bits = 0;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < n; base += stride) {
    const uint64_t v = base + (threadIdx.x & 31u);
    unsigned long long nb = 0;
    if (v < n) {
      nb = acc[v];
      fnext[v] = nb;
      if (nb) {
        seen[v] |= nb;
        acc[v] = 0ull;
      }
    }
    if (levels) {
      const unsigned int lo = __reduce_or_sync(0xffffffffu, (unsigned int)(nb & 0xffffffffull));
      const unsigned int hi = __reduce_or_sync(0xffffffffu, (unsigned int)(nb >> 32));
      unsigned long long any = ((unsigned long long)hi << 32) | lo;
      while (any) {
        const int j = __ffsll(any) - 1;
        any &= any - 1;
        if ((nb >> j) & 1ull) levels[(uint64_t)j * n + v] = next_level;
      }
    }
    found_v += nb != 0ull;
    found_bits += __popcll(nb);
    any_bits |= nb;
  }
  {
    const unsigned int lo = __reduce_or_sync(0xffffffffu, (unsigned int)(any_bits & 0xffffffffull));
    const unsigned int hi = __reduce_or_sync(0xffffffffu, (unsigned int)(any_bits >> 32));
    any_bits = ((unsigned long long)hi << 32) | lo;
  }
  for (int o = 16; o > 0; o >>= 1) {
    found_v += __shfl_xor_sync(0xffffffffu, found_v, o);
    found_bits += __shfl_xor_sync(0xffffffffu, found_bits, o);
  }
  if ((threadIdx.x & 31u) == 0) {
    if (found_v) atomicAdd(counters, found_v);
    if (found_bits) atomicAdd(counters + 1, found_bits);
    if (any_bits && live) atomicOr(live, any_bits);
  }
}

}  // namespace ms
}  // namespace gre
