// The 64-sources-per-word BFS (gre_msbfs) as one persistent launch.
//
// The level loop of the batched BFS (per level: a frontier list, a push or a pull, a commit of the
// new frontier words, and a host read of the counters that decides the next level's direction
// and whether to stop) runs inside one cooperative kernel: every block stays resident, the
// phases of a level are separated by a grid barrier, and the decisions are made by every block
// from the same counters in device memory.  The host launches once per 64-source word and reads
// the counters once at the end.  Per level:
//   phase A: push (a warp per frontier vertex, 64-bit atomicOr into acc) when the frontier's
//            out-arcs are fewer than m/14, else pull over the degree bins of the in-arcs (the
//            vertices' unseen sources among the live ones, early exit when all are found);
//   barrier;
//   phase B: commit acc into the next frontier and seen words, write the levels, append the new
//            frontier vertices to the next list with their out-degrees, count the new bits and
//            OR them into the next live mask;
//   barrier; stop when no bit was found.
// The results are those of the host-driven loop (same direction rule, same words), bit for bit.
//
// Waits.  A barrier waits on a generation counter with a time budget (GRE_GRID_WAIT_MS,
// default 2000 ms; 0 fails every wait at once, which the tests use).  A wait that runs out sets
// an error flag and returns; every block that sees the flag returns at its next barrier, so the
// kernel ends within about two budgets, the context stays usable, and the call returns
// GRE_TIMEOUT.  The launch is cooperative (cudaLaunchCooperativeKernel with at most the resident
// block count), so every block the barrier waits for is running.
//
// Memory that one phase writes and the next reads (frontier words, seen, acc, the lists and the
// counters) is read through L2 (ld.cg / volatile), never through the non-coherent L1 or the
// read-only path; the graph's arrays are read-only and use __ldg.
#include <algorithm>
#include <cstdlib>

#include "gre_internal.cuh"

namespace gre {

struct MsSlot {
  unsigned int nlist;          // frontier vertices in the list
  unsigned int pad0;
  unsigned long long arcs;     // their out-arcs
  unsigned long long found_v;  // vertices with new bits
  unsigned long long found_bits;
  unsigned long long live;     // OR of the new bits (sources that are still expanding)
  unsigned long long pad[3];
};

struct MsCtl {
  MsSlot slot[2];
  unsigned int bar_count, bar_gen, err, levels;
  unsigned long long push_levels, push_list, push_arcs, pull_levels, pull_scanned;
  unsigned long long pad[3];
};

constexpr int kMaxRecorded = GRE_MAX_RECORDED_SUPERSTEPS;

struct MsPersist {
  uint64_t n, m;
  const uint64_t* __restrict__ off;
  const uint32_t* __restrict__ col;
  const uint64_t* __restrict__ roff;
  const uint32_t* __restrict__ rcol;
  const uint32_t* __restrict__ rows;  // degree bins of the in-arcs
  uint64_t bin_start[DegreeBins::NB], bin_count[DegreeBins::NB];
  unsigned long long* seen;
  unsigned long long* fa;
  unsigned long long* fb;
  unsigned long long* acc;
  uint32_t* list0;
  uint32_t* list1;
  int32_t* levels;                     // k rows of n int32 (this word's sources)
  unsigned long long* found_per_level; // kMaxRecorded entries
  MsCtl* ctl;
  long long wait_ns;
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <class T>
__device__ __forceinline__ T vload(const T* p) {
  return *(const volatile T*)p;
}

// Grid barrier with a bounded wait (see the file comment).  Returns false when the kernel must
// end (a wait ran out here or in another block).
__device__ bool grid_sync(MsCtl* c, long long wait_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    if (vload(&c->err)) {
      ok = 0;
    } else {
      const unsigned int gen = vload(&c->bar_gen);
      __threadfence();
      const unsigned int arrived = atomicAdd(&c->bar_count, 1u) + 1u;
      if (arrived == gridDim.x) {
        atomicExch(&c->bar_count, 0u);
        __threadfence();
        atomicAdd(&c->bar_gen, 1u);
      } else {
        const unsigned long long t0 = globaltimer_ns();
        for (;;) {
          if (wait_ns == 0 || (long long)(globaltimer_ns() - t0) >= wait_ns) {
            atomicOr(&c->err, 1u);
            ok = 0;
            break;
          }
          if (vload(&c->bar_gen) != gen) break;
          if (vload(&c->err)) {
            ok = 0;
            break;
          }
          __nanosleep(100);
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Pull over the rows of one bin with L lanes per row (L <= 16): acc[v] = (OR of the in-neighbours'
// frontier words) & live & ~seen[v]; a lone lane stops once every wanted source is found.
template <int L>
__device__ void pull_small(const MsPersist& P, const uint32_t* rows, uint64_t count, unsigned long long live,
                           const unsigned long long* fd, uint64_t gwarp, uint64_t nwarps, unsigned long long* scanned) {
  constexpr int G = 32 / L;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lig = lane % L;
  for (uint64_t base = gwarp * G; base < count; base += nwarps * G) {
    const uint64_t i = base + lane / L;
    unsigned long long got = 0, want = 0;
    uint32_t v = 0;
    if (i < count) {
      v = __ldg(rows + i);
      want = live & ~__ldcg(P.seen + v);
      if (want) {
        const uint64_t a1 = __ldg(P.roff + v + 1);
        for (uint64_t a = __ldg(P.roff + v) + lig; a < a1; a += L) {
          got |= __ldcg(fd + __ldg(P.rcol + a));
          ++*scanned;
          if (L == 1 && (got & want) == want) break;
        }
      }
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) got |= __shfl_xor_sync(0xffffffffu, got, o);
    if (i < count && lig == 0 && (got & want)) P.acc[v] = got & want;
  }
}

// Rows of more than the small bins' arcs: a warp per row, the warp stops when its lanes' OR covers
// every wanted source.
__device__ void pull_long(const MsPersist& P, const uint32_t* rows, uint64_t count, unsigned long long live,
                          const unsigned long long* fd, uint64_t gwarp, uint64_t nwarps, unsigned long long* scanned) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t i = gwarp; i < count; i += nwarps) {
    const uint32_t v = __ldg(rows + i);
    const unsigned long long want = live & ~__ldcg(P.seen + v);
    if (!want) continue;  // uniform: one row per warp
    unsigned long long got = 0;
    const uint64_t a0 = __ldg(P.roff + v), a1 = __ldg(P.roff + v + 1);
    for (uint64_t b = a0; b < a1; b += 32) {
      if (b + lane < a1) {
        got |= __ldcg(fd + __ldg(P.rcol + b + lane));
        ++*scanned;
      }
      const unsigned int lo = __reduce_or_sync(0xffffffffu, (unsigned int)(got & 0xffffffffull));
      const unsigned int hi = __reduce_or_sync(0xffffffffu, (unsigned int)(got >> 32));
      got = ((unsigned long long)hi << 32) | lo;
      if ((got & want) == want) break;
    }
    if (lane == 0 && (got & want)) P.acc[v] = got & want;
  }
}

__global__ void __launch_bounds__(256) k_msbfs_persist(MsPersist P) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t gwarp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  MsCtl* c = P.ctl;
  unsigned long long* front = P.fa;
  unsigned long long* next = P.fb;
  for (int32_t d = 0;; ++d) {
    const int cur = d & 1, prev = cur ^ 1;
    const MsSlot* ps = &c->slot[prev];  // the frontier of level d (committed by level d-1)
    const unsigned long long nlist = vload(&ps->nlist);
    const unsigned long long farcs = vload(&ps->arcs);
    const unsigned long long live = vload(&ps->live);
    const uint32_t* list = prev ? P.list1 : P.list0;
    const bool push = farcs * 14 < P.m;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      MsSlot* cs = &c->slot[cur];  // last read two barriers ago: free for this level's counts
      cs->nlist = 0;
      cs->arcs = 0;
      cs->found_v = 0;
      cs->found_bits = 0;
      cs->live = 0;
      if (push) {
        c->push_levels += 1;
        c->push_list += nlist;
        c->push_arcs += farcs;
      } else {
        c->pull_levels += 1;
      }
      __threadfence();
    }
    // phase A
    unsigned long long scanned = 0;
    if (push) {
      for (uint64_t i = gwarp; i < nlist; i += nwarps) {
        const uint32_t u = __ldcg(list + i);
        const unsigned long long fu = __ldcg(front + u);
        const uint64_t a1 = __ldg(P.off + u + 1);
        for (uint64_t a = __ldg(P.off + u) + lane; a < a1; a += 32) {
          const uint32_t v = __ldg(P.col + a);
          const unsigned long long bits = fu & ~__ldcg(P.seen + v);
          if (bits && (__ldcg(P.acc + v) & bits) != bits) atomicOr(P.acc + v, bits);
        }
      }
    } else {
      pull_small<1>(P, P.rows + P.bin_start[0], P.bin_count[0], live, front, gwarp, nwarps, &scanned);
      pull_small<2>(P, P.rows + P.bin_start[1], P.bin_count[1], live, front, gwarp, nwarps, &scanned);
      pull_small<4>(P, P.rows + P.bin_start[2], P.bin_count[2], live, front, gwarp, nwarps, &scanned);
      pull_small<8>(P, P.rows + P.bin_start[3], P.bin_count[3], live, front, gwarp, nwarps, &scanned);
      pull_small<16>(P, P.rows + P.bin_start[4], P.bin_count[4], live, front, gwarp, nwarps, &scanned);
      pull_long(P, P.rows + P.bin_start[5], P.bin_count[5] + P.bin_count[6] + P.bin_count[7], live, front, gwarp, nwarps,
                &scanned);
      for (int o = 16; o > 0; o >>= 1) scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
      if (lane == 0 && scanned) atomicAdd(&c->pull_scanned, scanned);
    }
    if (!grid_sync(c, P.wait_ns)) return;
    // phase B: commit
    MsSlot* cs = &c->slot[cur];
    uint32_t* nlist_out = cur ? P.list1 : P.list0;
    unsigned long long found_v = 0, found_bits = 0, any_bits = 0, deg = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < P.n; base += stride) {
      const uint64_t v = base + lane;
      unsigned long long nb = 0;
      if (v < P.n) {
        nb = __ldcg(P.acc + v);
        next[v] = nb;
        if (nb) {
          P.seen[v] = __ldcg(P.seen + v) | nb;
          P.acc[v] = 0ull;
          deg += __ldg(P.off + v + 1) - __ldg(P.off + v);
        }
      }
      const unsigned int lo = __reduce_or_sync(0xffffffffu, (unsigned int)(nb & 0xffffffffull));
      const unsigned int hi = __reduce_or_sync(0xffffffffu, (unsigned int)(nb >> 32));
      unsigned long long any = ((unsigned long long)hi << 32) | lo;
      any_bits |= any;
      while (any) {
        const int j = __ffsll(any) - 1;
        any &= any - 1;
        if ((nb >> j) & 1ull) P.levels[(uint64_t)j * P.n + v] = d + 1;
      }
      const uint32_t pos = warp_append(&cs->nlist, nb != 0ull);
      if (nb) nlist_out[pos] = (uint32_t)v;
      found_v += nb != 0ull;
      found_bits += __popcll(nb);
    }
    for (int o = 16; o > 0; o >>= 1) {
      found_v += __shfl_xor_sync(0xffffffffu, found_v, o);
      found_bits += __shfl_xor_sync(0xffffffffu, found_bits, o);
      deg += __shfl_xor_sync(0xffffffffu, deg, o);
    }
    if (lane == 0) {
      if (found_v) atomicAdd(&cs->found_v, found_v);
      if (found_bits) atomicAdd(&cs->found_bits, found_bits);
      if (deg) atomicAdd(&cs->arcs, deg);
      if (any_bits) atomicOr(&cs->live, any_bits);
    }
    if (!grid_sync(c, P.wait_ns)) return;
    const unsigned long long fb = vload(&cs->found_bits);
    if (blockIdx.x == 0 && threadIdx.x == 0 && d < kMaxRecorded) P.found_per_level[d] = fb;
    if (fb == 0) {
      if (blockIdx.x == 0 && threadIdx.x == 0) c->levels = (unsigned int)d;
      return;
    }
    unsigned long long* t = front;
    front = next;
    next = t;
  }
}

// frontier list of level 0 (the sources' vertices, each once) and its out-arcs
__global__ void k_ms_first_list(uint64_t n, const unsigned long long* __restrict__ f, const uint64_t* __restrict__ off,
                                uint32_t* __restrict__ list, MsSlot* __restrict__ s) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long deg = 0;
  for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) & ~31ull; base < n; base += stride) {
    const uint64_t v = base + (threadIdx.x & 31u);
    const bool nz = v < n && f[v] != 0ull;
    const uint32_t pos = warp_append(&s->nlist, nz);
    if (nz) {
      list[pos] = (uint32_t)v;
      deg += off[v + 1] - off[v];
    }
  }
  for (int o = 16; o > 0; o >>= 1) deg += __shfl_xor_sync(0xffffffffu, deg, o);
  if ((threadIdx.x & 31u) == 0 && deg) atomicAdd(&s->arcs, deg);
}

// Budget of a grid-barrier wait in ns (GRE_GRID_WAIT_MS; default 2000 ms).
static long long grid_wait_ns() {
  if (const char* e = getenv("GRE_GRID_WAIT_MS")) return (long long)strtoll(e, nullptr, 10) * 1000000ll;
  return 2000ll * 1000000ll;
}

// Whether the persistent form runs for a graph of n vertices: by default below 2^23 vertices,
// where the host loop's per-level launches and counter reads are a visible share of a level
// (RMAT-20, 64 sources: 2.82 against 2.92 ms); above, the resident grid (fewer blocks per SM than
// the separate kernels) made it slower (RMAT-26: 88.5 against 85.8 ms).  GRE_PERSIST=1 / 0
// forces it on / off.  Needs a device that can launch cooperatively.
bool msbfs_persistent_available(uint64_t n) {
  if (const char* e = getenv("GRE_PERSIST")) {
    if (strtoul(e, nullptr, 10) == 0) return false;
  } else if (n >= (1ull << 23)) {
    return false;
  }
  int dev = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess) return false;
  return coop != 0;
}

// One 64-source word from the seeded state (seen, fa = the sources' words, levels row 0 set):
// the whole level loop in one cooperative launch.  Adds the level statistics to the outputs.
int msbfs_word_persistent(gre_graph g, unsigned long long full, unsigned long long* seen, unsigned long long* fa,
                          unsigned long long* fb, unsigned long long* acc, uint32_t* list0, uint32_t* list1, int32_t* levels,
                          void* ctl_mem, unsigned long long* found_per_level, uint32_t* levels_out, uint64_t* scanned,
                          uint64_t* bytes, std::vector<unsigned long long>* found) {
  const uint64_t n = g->n;
  MsCtl* ctl = (MsCtl*)ctl_mem;
  GRE_CUDA(cudaMemsetAsync(ctl, 0, sizeof(MsCtl), g->stream));
  GRE_CUDA(cudaMemcpyAsync(&ctl->slot[1].live, &full, sizeof full, cudaMemcpyHostToDevice, g->stream));
  k_ms_first_list<<<grid_for(n, 256, 8), 256, 0, g->stream>>>(n, fa, g->off, list1, &ctl->slot[1]);
  GRE_LAUNCH_CHECK();
  static int per_sm = 0;
  if (!per_sm) {
    int b = 0;
    GRE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_msbfs_persist, 256, 0));
    per_sm = b > 0 ? b : 1;
  }
  const DegreeBins& B = g->bins_in;
  MsPersist P;
  P.n = n;
  P.m = g->m;
  P.off = g->off;
  P.col = g->col;
  P.roff = g->roff;
  P.rcol = g->rcol;
  P.rows = B.rows;
  for (int b = 0; b < DegreeBins::NB; ++b) {
    P.bin_start[b] = B.start[b];
    P.bin_count[b] = B.count[b];
  }
  P.seen = seen;
  P.fa = fa;
  P.fb = fb;
  P.acc = acc;
  P.list0 = list0;
  P.list1 = list1;
  P.levels = levels;
  P.found_per_level = found_per_level;
  P.ctl = ctl;
  P.wait_ns = grid_wait_ns();
  void* args[] = {&P};
  const int grid = num_sms() * per_sm;
  GRE_CUDA(cudaLaunchCooperativeKernel((const void*)k_msbfs_persist, dim3(grid), dim3(256), args, 0, g->stream));
  MsCtl h;
  GRE_CUDA(cudaMemcpyAsync(&h, ctl, sizeof h, cudaMemcpyDeviceToHost, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  if (h.err) {
    set_error("gre_msbfs: a grid barrier wait of the persistent level loop ran out (%lld ms budget)",
              (long long)(P.wait_ns / 1000000ll));
    return GRE_TIMEOUT;
  }
  *levels_out = h.levels;
  *scanned += h.push_arcs + h.pull_scanned;
  *bytes += 16 * h.push_list + 12 * h.push_arcs + 32 * n * h.push_levels + 24 * n * h.pull_levels + 12 * h.pull_scanned;
  if (found) {
    const uint32_t k = std::min<uint32_t>(h.levels + 1, kMaxRecorded);
    found->resize(k);
    GRE_CUDA(cudaMemcpy(found->data(), found_per_level, sizeof(unsigned long long) * k, cudaMemcpyDeviceToHost));
  }
  return GRE_SUCCESS;
}

size_t msbfs_ctl_bytes() { return sizeof(MsCtl) + sizeof(unsigned long long) * kMaxRecorded; }

}  // namespace gre
