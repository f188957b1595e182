// The reference plugins as device VertexCode plugins (gre/vertex_code.cuh).  Each callback
// restates the reference callback of the same name; only the locking of combine changes (an
// atomic instead of the striped spin lock), which keeps the combine semantics.
#pragma once
#include <stdint.h>

#include "../../include/gre/vertex_code.cuh"

namespace gre {

// output_statistics helpers: fixed-shape reductions, so a sum is the same bits on every run.
namespace plugin_stats {
constexpr int kBlocks = 256, kThreads = 256;
// per-block sums of x[0..n) into partial[0..kBlocks), then their sum into partial[kBlocks]
__global__ void __launch_bounds__(kThreads) k_sum_f64(const double* __restrict__ x, uint64_t n, double* __restrict__ partial) {
  __shared__ double s[kThreads];
  double a = 0.0;
  for (uint64_t v = blockIdx.x * (uint64_t)kThreads + threadIdx.x; v < n; v += (uint64_t)kBlocks * kThreads) a += x[v];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}
__global__ void k_sum_partials(double* partial) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double a = 0.0;
  for (int b = 0; b < kBlocks; ++b) a += partial[b];
  partial[kBlocks] = a;
}
// number of v with lab[v] == vid(v) (CC.hpp:80-94), or the sum of cnt[v] (CountIn.hpp:78-86)
__global__ void k_count(uint64_t n, const uint32_t* __restrict__ lab, const uint32_t* __restrict__ vid,
                        const int32_t* __restrict__ cnt, unsigned long long* __restrict__ out) {
  unsigned long long a = 0;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    a += lab ? (lab[v] == (vid ? vid[v] : (uint32_t)v) ? 1ull : 0ull) : (unsigned long long)cnt[v];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31u) == 0 && a) atomicAdd(out, a);
}

// Host side: run one reduction on the engine's stream and store it in *out_value / *out_count.
inline void sum_f64(const EngineContext& ctx, const double* x, double* scratch, double* out_value) {
  if (!out_value) return;
  k_sum_f64<<<kBlocks, kThreads, 0, ctx.stream>>>(x, ctx.n, scratch);
  k_sum_partials<<<1, 32, 0, ctx.stream>>>(scratch);
  cudaMemcpyAsync(out_value, scratch + kBlocks, sizeof(double), cudaMemcpyDeviceToHost, ctx.stream);
  cudaStreamSynchronize(ctx.stream);
}
inline void count(const EngineContext& ctx, const uint32_t* lab, const uint32_t* vid, const int32_t* cnt, double* scratch,
                  uint64_t* out_count) {
  if (!out_count) return;
  unsigned long long* d = (unsigned long long*)scratch;
  unsigned long long h = 0;
  cudaMemsetAsync(d, 0, sizeof h, ctx.stream);
  k_count<<<kBlocks, kThreads, 0, ctx.stream>>>(ctx.n, lab, vid, cnt, d);
  cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, ctx.stream);
  cudaStreamSynchronize(ctx.stream);
  *out_count = h;
}
}  // namespace plugin_stats

// PageRank (Kernels/PageRank.hpp:38-79).  refresh=false is the reference verbatim (pr_scatter
// is set in init only); refresh=true is PageRankIter (pr_scatter = pr/outdeg in apply).
struct VcPageRank {
  typedef double msg_t;
  double* pr;
  double* scat;
  double* comb;
  const uint32_t* outdeg;
  double tele;  // 0.15 in the reference (dampingFactor, PageRank.hpp:20)
  double d;     // 1 - 0.15
  bool refresh;
  double* stat_scratch = nullptr;  // device, plugin_stats::kBlocks + 1 doubles
  double* stat_sum = nullptr;      // host: output_statistics' sum of pr (null: not reported)
  __device__ bool init(uint32_t v) {
    pr[v] = tele;
    const uint32_t od = outdeg[v];
    if (od > 0) {
      scat[v] = pr[v] / (double)od;
      return true;
    }
    return false;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  __device__ bool combine(uint32_t v, const double& m) {
    atomicAdd(comb + v, m);
    return true;
  }
  __device__ bool apply(uint32_t v) {
    pr[v] = tele + d * comb[v];
    comb[v] = 0.0;
    if (refresh) {
      const uint32_t od = outdeg[v];
      if (od > 0) scat[v] = pr[v] / (double)od;
    }
    return false;
  }
  __device__ bool assert_to_halt(uint32_t) { return false; }
  void reduce() {}
  // "Sum of pr" (PageRank.hpp:102-124; the agent and edge counts it also prints are 0 and m at
  // one rank)
  void output_statistics(const EngineContext& ctx) { plugin_stats::sum_f64(ctx, pr, stat_scratch, stat_sum); }
};

// BFS (Kernels/BFS.hpp:34-72): parent tree, first writer wins.  `level` (optional) records the
// superstep in which apply fixed the parent, i.e. the depth in the tree.
struct VcBFS {
  typedef unsigned long long msg_t;
  unsigned long long* pred;
  unsigned long long* scat;
  unsigned long long* comb;
  int32_t* level;
  const uint32_t* vid;  // get_vid (DistributedGraph.hpp:57-59): internal -> caller id, null = identity
  int32_t cur = 0;      // superstep index, advanced by reduce()
  __device__ bool init(uint32_t v) {
    pred[v] = vid ? vid[v] : v;  // pred[lv] = graph.get_vid(lv)
    scat[v] = pred[v];
    if (level) level[v] = 0;
    return true;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  __device__ bool combine(uint32_t v, const msg_t& m) {
    if (comb[v] != ~0ull) return false;  // the reference's unlocked pre-check
    return atomicCAS(comb + v, ~0ull, m) == ~0ull;
  }
  __device__ bool apply(uint32_t v) {
    if (pred[v] == ~0ull) {
      pred[v] = comb[v];
      scat[v] = pred[v];
      if (level) level[v] = cur + 1;
      return true;
    }
    return false;
  }
  __device__ bool assert_to_halt(uint32_t) { return true; }
  void reduce() { ++cur; }
};

// SSSP (Kernels/SSSP.hpp:55-89) with a uint32 weight per CSR arc.
struct VcSSSP {
  typedef uint32_t msg_t;
  uint32_t* states;
  uint32_t* last;
  const uint32_t* w;
  __device__ bool init(uint32_t v) {
    states[v] = 0;
    last[v] = 0;
    return true;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t arc) { ctx.sendMessage(v, last[u] + w[arc]); }
  __device__ bool combine(uint32_t v, const uint32_t& m) {
    if (!(m < states[v])) return false;
    return atomicMin(states + v, m) > m;
  }
  __device__ bool apply(uint32_t v) {
    last[v] = states[v];
    return true;
  }
  __device__ bool assert_to_halt(uint32_t) { return true; }
  void reduce() {}
};

// PageRank_delta (Kernels/PageRank.hpp:129-197): only the change of a vertex's rank travels; a
// vertex stays active while its change exceeds err.
struct VcPageRankDelta {
  typedef double msg_t;
  double* pr;
  double* scat;
  double* comb;
  const uint32_t* outdeg;
  double tele;  // dampingFactor = 0.15 (PageRank.hpp:131)
  double d;     // 1 - 0.15
  double err;   // 1e-5 (PageRank.hpp:132)
  __device__ bool init(uint32_t v) {
    pr[v] = tele;
    const uint32_t od = outdeg[v];
    if (od > 0) {
      scat[v] = pr[v] / (double)od;
      return true;
    }
    return false;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  __device__ bool combine(uint32_t v, const double& m) {
    atomicAdd(comb + v, m);
    return true;
  }
  __device__ bool apply(uint32_t v) {
    const double delta = d * comb[v];
    pr[v] += delta;
    comb[v] = 0.0;
    const uint32_t od = outdeg[v];
    if (delta > err && od > 0) {
      scat[v] = delta / (double)od;
      return true;
    }
    return false;
  }
  __device__ bool assert_to_halt(uint32_t) { return true; }
  void reduce() {}
};

// SSSP with predecessors (Kernels/SSSP1.hpp:62-95).  A state packs (dist << 32 | pred), pred a
// caller vertex id, so one 64-bit atomicMin keeps the pair consistent.  combine reports an
// improvement only when the distance drops (a tie with a smaller pred updates pred without
// activating the vertex), so the active sets equal the reference's; among senders at equal
// distance the reference keeps whichever message arrived first, this keeps the smallest id.
struct VcSSSP1 {
  typedef unsigned long long msg_t;
  unsigned long long* states;
  uint32_t* last;
  const uint32_t* w;
  const uint32_t* vid;  // get_vid: internal -> caller id, null = identity
  __device__ bool init(uint32_t v) {
    const unsigned long long me = vid ? vid[v] : v;
    states[v] = me;  // dist 0, pred = self
    last[v] = 0;
    return true;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t arc) {
    const uint32_t dist = last[u] + w[arc];
    ctx.sendMessage(v, ((unsigned long long)dist << 32) | (vid ? vid[u] : u));
  }
  __device__ bool combine(uint32_t v, const unsigned long long& m) {
    if (!(m < states[v])) return false;
    const unsigned long long old = atomicMin(states + v, m);
    return (uint32_t)(m >> 32) < (uint32_t)(old >> 32);
  }
  __device__ bool apply(uint32_t v) {
    last[v] = (uint32_t)(states[v] >> 32);
    return true;
  }
  __device__ bool assert_to_halt(uint32_t) { return true; }
  void reduce() {}
};

// CountIn (Kernels/CountIn.hpp:33-56): every vertex sends 1 along its arcs of the run's
// direction; apply stores the count received.  One superstep in the reference driver.
struct VcCountIn {
  typedef int32_t msg_t;
  int32_t* cn;
  int32_t* scat;
  int32_t* comb;
  double* stat_scratch = nullptr;  // device, one 8-byte counter
  uint64_t* stat_count = nullptr;  // host: output_statistics' "Number of in edges" (null: not reported)
  __device__ bool init(uint32_t v) {
    cn[v] = 0;
    scat[v] = 1;
    return true;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  __device__ bool combine(uint32_t v, const int32_t& m) {
    atomicAdd(comb + v, m);
    return true;
  }
  __device__ bool apply(uint32_t v) {
    cn[v] = comb[v];
    return false;
  }
  __device__ bool assert_to_halt(uint32_t) { return true; }
  void reduce() {}
  // "Number of in edges": the sum of the counts (CountIn.hpp:78-100)
  void output_statistics(const EngineContext& ctx) { plugin_stats::count(ctx, nullptr, nullptr, cn, stat_scratch, stat_count); }
};

// ConnectedComponents (Kernels/CC.hpp:33-67): min-vid label propagation.  Labels are vids,
// stored as uint32 (every vid fits).
struct VcCC {
  typedef uint32_t msg_t;
  uint32_t* cc;
  uint32_t* scat;
  uint32_t* comb;
  const uint32_t* vid;  // get_vid: internal -> caller id, null = identity
  double* stat_scratch = nullptr;  // device, one 8-byte counter
  uint64_t* stat_count = nullptr;  // host: the number of components (null: not reported)
  __device__ bool init(uint32_t v) {
    cc[v] = vid ? vid[v] : v;  // cc[lv] = graph.get_vid(lv)
    scat[v] = cc[v];
    comb[v] = cc[v];
    return true;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  __device__ bool combine(uint32_t v, const uint32_t& m) {
    if (!(comb[v] > m)) return false;
    return atomicMin(comb + v, m) > m;
  }
  __device__ bool apply(uint32_t v) {
    if (comb[v] >= cc[v]) return false;
    cc[v] = comb[v];
    scat[v] = cc[v];
    return true;
  }
  __device__ bool assert_to_halt(uint32_t) { return true; }
  void reduce() {}
  // "Number of components" (CC.hpp:73-120 prints it from reduce every superstep; the value
  // after the last superstep is the one reported here)
  void output_statistics(const EngineContext& ctx) { plugin_stats::count(ctx, cc, vid, nullptr, stat_scratch, stat_count); }
};

// BC Forward (Kernels/BC.hpp:56-91): level and path count; numPaths is FP64 here (the
// reference's int32 wraps on large graphs; values agree below 2^31).
struct VcForward {
  typedef double msg_t;
  int32_t* level;
  double* sigma;
  double* scat;
  double* sum;
  int32_t currLevel = 1;
  __device__ bool init(uint32_t v) {
    sigma[v] = 1.0;
    level[v] = 0;
    scat[v] = 1.0;
    return true;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  __device__ bool combine(uint32_t v, const double& m) {
    atomicAdd(sum + v, m);
    return true;
  }
  __device__ bool apply(uint32_t v) {
    if (level[v] < 0) {
      level[v] = currLevel;
      sigma[v] = sum[v];
      scat[v] = sigma[v];
      return true;
    }
    return false;
  }
  __device__ bool assert_to_halt(uint32_t) { return true; }
  void reduce() { ++currLevel; }
};

// BC Backward (Kernels/BC.hpp:132-163): one superstep per level; `sum` is kept across levels.
struct VcBackward {
  typedef double msg_t;
  const int32_t* level;
  const double* sigma;
  double* dep;
  double* pathwgt;
  double* sum;
  int32_t currLevel = 0;
  __device__ bool init(uint32_t v) {
    if (level[v] == currLevel) {
      pathwgt[v] = (1.0 + dep[v]) / sigma[v];
      return true;
    }
    return false;
  }
  template <class Ctx>
  __device__ void scatter(Ctx& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, pathwgt[u]); }
  __device__ bool combine(uint32_t v, const double& m) {
    atomicAdd(sum + v, m);
    return true;
  }
  __device__ bool apply(uint32_t v) {
    if (level[v] == currLevel - 1) dep[v] = sum[v] * sigma[v];
    return false;
  }
  __device__ bool assert_to_halt(uint32_t) { return true; }
  void reduce() {}
};

}  // namespace gre
