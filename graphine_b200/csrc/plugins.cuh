// The reference plugins as device VertexCode plugins (gre/vertex_code.cuh).  Each callback
// restates the reference callback of the same name; only the locking of combine changes (an
// atomic instead of the striped spin lock), which keeps the combine semantics.
#pragma once
#include <stdint.h>

#include "../../include/gre/vertex_code.cuh"

namespace gre {

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
};

// ConnectedComponents (Kernels/CC.hpp:33-67): min-vid label propagation.  Labels are vids,
// stored as uint32 (every vid fits).
struct VcCC {
  typedef uint32_t msg_t;
  uint32_t* cc;
  uint32_t* scat;
  uint32_t* comb;
  const uint32_t* vid;  // get_vid: internal -> caller id, null = identity
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
