// ORACLE — test infrastructure only (CPU restatement of the reference's hot path).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this library,
// and only as the checker.  The product (graphine_b200/, include/) never links or calls it.
//
// What is restated, np = 1 (one rank owns every vertex, lvid == vid):
//   * loader: `<prefix>.meta` + `<prefix>.edges.<i>`        Graph/GraphIngress.hpp:323-328,511-723
//     CSR in source-major / input order                       Graph/LocalGraph.hpp:66-107
//     reverse CSR + redgeID (arc id of each reverse slot)     Graph/LocalGraph.hpp:112-156
//     outdegree = number of lines with that source            Graph/GraphIngress.hpp:591
//   * the BSP superstep loop of SynchronousEngine::run_master / fn_worker_tp
//     init (all or sources)                                   Engine/Engine.hpp:437-471
//     compute: every active vertex scatters along its arcs; sendMessage = combine, and on
//     success the destination's bit in nextSet is set       Engine/Engine.hpp:592-625,1384-1389
//     assert_to_halt after scattering                         Engine/Engine.hpp:619-623
//     apply only for vertices whose nextSet bit is set; a true return re-activates the vertex;
//     the active list is rebuilt from the bitmap              Engine/Engine.hpp:760-798
//     vertexCode.reduce(); stop when no vertex is active      Engine/Engine.hpp:386-400
//     superstep count is not incremented on that break        Engine/Engine.hpp:269,399-400
//   * the plugins: PageRank (Kernels/PageRank.hpp:38-79), BFS (Kernels/BFS.hpp:34-72),
//     SSSP (Kernels/SSSP.hpp:55-89) with the harness weights, ConnectedComponents
//     (Kernels/CC.hpp:33-67), BC Forward/Backward (Kernels/BC.hpp:56-163) and the BC driver
//     loop (usr/test_bc.cpp:63-110).
//   * harness plugins written against the same contract: PageRankIter (PageRank + the
//     pr_scatter refresh the reference leaves out), personalised PageRank, and the weighted
//     PageRank forward/adjoint used for the gradient checks (no reference counterpart).
//
// Direction In: the reference indexes the reverse arc list with the forward offsets
// (LocalGraph.hpp:183-191).  That is the same as the true reverse offsets whenever in-degree
// equals out-degree, i.e. on the symmetric graphs every run<In> of the drivers sees; this
// restatement uses the true reverse offsets.
//
// The restatement is sequential (one thread per independent run); the per-vertex order in
// which messages are combined is therefore fixed, and integer results do not depend on it.
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "oracle_common.hpp"

namespace {

enum { DIR_OUT = 0, DIR_IN = 1, DIR_INOUT = 2 };

struct OGraph {
  uint64_t n = 0, m = 0;
  std::vector<uint64_t> off, roff;  // forward and reverse offsets
  std::vector<uint32_t> col, rcol;  // forward and reverse neighbour lists
  std::vector<uint64_t> rarc;       // reverse slot -> forward arc id (redgeID)
  std::vector<int64_t> outdeg;
};

void build(OGraph* g, const std::vector<uint32_t>& src, const std::vector<uint32_t>& dst) {
  const uint64_t n = g->n, m = src.size();
  g->m = m;
  g->off.assign(n + 1, 0);
  g->roff.assign(n + 1, 0);
  for (uint64_t i = 0; i < m; ++i) {
    g->off[src[i] + 1]++;
    g->roff[dst[i] + 1]++;
  }
  for (uint64_t v = 0; v < n; ++v) {
    g->off[v + 1] += g->off[v];
    g->roff[v + 1] += g->roff[v];
  }
  g->col.resize(m);
  g->rcol.resize(m);
  g->rarc.resize(m);
  std::vector<uint64_t> cur(g->off.begin(), g->off.end() - 1);
  std::vector<uint64_t> arc_of_edge(m);
  for (uint64_t i = 0; i < m; ++i) {
    arc_of_edge[i] = cur[src[i]];
    g->col[cur[src[i]]++] = dst[i];
  }
  std::vector<uint64_t> rcur(g->roff.begin(), g->roff.end() - 1);
  for (uint64_t i = 0; i < m; ++i) {
    const uint64_t s = rcur[dst[i]]++;
    g->rcol[s] = src[i];
    g->rarc[s] = arc_of_edge[i];
  }
  g->outdeg.assign(n, 0);
  for (uint64_t v = 0; v < n; ++v) g->outdeg[v] = (int64_t)(g->off[v + 1] - g->off[v]);
}

// ----------------------------------------------------------------------------------------------
// The superstep loop.
// ----------------------------------------------------------------------------------------------
struct Trace {
  std::vector<uint64_t> active;  // active vertices after each superstep
  uint32_t supersteps = 0;
};

template <class VC>
struct Ctx {
  VC* vc;
  std::vector<uint8_t>* next;
  void sendMessage(uint32_t v, typename VC::msg_t msg) {
    if (vc->combine(v, msg)) (*next)[v] = 1;
  }
};

template <class VC>
void run(const OGraph& g, VC& vc, int dir, const uint32_t* srcs, uint32_t nsrc, uint32_t max_ss,
         Trace* tr) {
  const uint64_t n = g.n;
  std::vector<uint8_t> curr(n, 0), next(n, 0);
  std::vector<uint32_t> list;
  if (!srcs) {
    for (uint64_t v = 0; v < n; ++v)
      if (vc.init((uint32_t)v)) {
        curr[v] = 1;
        list.push_back((uint32_t)v);
      }
  } else {
    for (uint32_t i = 0; i < nsrc; ++i) {
      const uint32_t v = srcs[i];
      if (vc.init(v) && !curr[v]) {  // setAndInsert (Graph/VertexSet.hpp:128-134)
        curr[v] = 1;
        list.push_back(v);
      }
    }
  }
  Ctx<VC> ctx{&vc, &next};
  uint32_t ss = 0;
  for (ss = 0; ss < max_ss; ++ss) {
    vc.superstep = ss;
    std::fill(next.begin(), next.end(), 0);
    for (uint32_t u : list) {
      if (dir == DIR_OUT || dir == DIR_INOUT)
        for (uint64_t a = g.off[u]; a < g.off[u + 1]; ++a) vc.scatter(ctx, u, g.col[a], a);
      if (dir == DIR_IN || dir == DIR_INOUT)
        for (uint64_t a = g.roff[u]; a < g.roff[u + 1]; ++a) vc.scatter(ctx, u, g.rcol[a], g.rarc[a]);
      if (vc.assert_to_halt(u)) curr[u] = 0;
    }
    list.clear();
    for (uint64_t v = 0; v < n; ++v)
      if (next[v] && vc.apply((uint32_t)v)) curr[v] = 1;
    for (uint64_t v = 0; v < n; ++v)
      if (curr[v]) list.push_back((uint32_t)v);
    vc.reduce();
    if (tr) tr->active.push_back(list.size());
    if (list.empty()) break;
  }
  if (tr) tr->supersteps = ss;
}

// ----------------------------------------------------------------------------------------------
// Plugins.
// ----------------------------------------------------------------------------------------------
struct PluginBase {
  uint32_t superstep = 0;
  bool assert_to_halt(uint32_t) { return true; }  // VertexCode.hpp:50
  void reduce() {}
};

// PageRank (Kernels/PageRank.hpp:38-79) and the harness PageRankIter / personalised form.
// teleport[v] = (1-d)·w_v: the reference has d = 0.85 and w = 1 (dampingFactor = 0.15 at
// PageRank.hpp:20 is the teleport weight).  refresh = false reproduces the reference exactly:
// apply never refreshes pr_scatter, so every superstep re-sends the initial 0.15/outdeg.
struct PageRankVC : PluginBase {
  typedef double msg_t;
  const OGraph* g;
  double d;
  const double* teleport;  // null: 1-d for every vertex
  bool refresh;
  std::vector<double> pr, scat, comb;
  double tele(uint32_t v) const { return teleport ? teleport[v] : 1.0 - d; }
  bool init(uint32_t v) {
    pr[v] = tele(v);
    if (g->outdeg[v] > 0) {
      scat[v] = pr[v] / (double)g->outdeg[v];
      return true;
    }
    return false;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  bool combine(uint32_t v, double m) {
    comb[v] += m;
    return true;
  }
  bool apply(uint32_t v) {
    pr[v] = tele(v) + d * comb[v];
    comb[v] = 0.0;
    if (refresh && g->outdeg[v] > 0) scat[v] = pr[v] / (double)g->outdeg[v];
    return false;
  }
  bool assert_to_halt(uint32_t) { return false; }  // PageRank.hpp:77-79
};

// BFS parent tree (Kernels/BFS.hpp:34-72); level[] records the superstep of discovery, which
// equals the depth in the pred tree.
struct BFSVC : PluginBase {
  typedef uint64_t msg_t;
  std::vector<uint64_t> pred, scat, comb;
  std::vector<int32_t> level;
  bool init(uint32_t v) {
    pred[v] = v;
    scat[v] = v;
    level[v] = 0;
    return true;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  bool combine(uint32_t v, uint64_t m) {
    if (comb[v] == ~0ull) {
      comb[v] = m;
      return true;
    }
    return false;
  }
  bool apply(uint32_t v) {
    if (pred[v] == ~0ull) {
      pred[v] = comb[v];
      scat[v] = pred[v];
      level[v] = (int32_t)superstep + 1;
      return true;
    }
    return false;
  }
};

// SSSP (Kernels/SSSP.hpp:55-89), weight = harness weight of the arc's endpoints or a given
// per-arc weight array (forward CSR order).
struct SSSPVC : PluginBase {
  typedef uint32_t msg_t;
  std::vector<uint32_t> states, last;
  uint64_t wseed;
  const uint32_t* warc;
  bool init(uint32_t v) {
    states[v] = 0;
    last[v] = 0;
    return true;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t arc) {
    const uint32_t w = warc ? warc[arc] : gre_oracle::sssp_weight(wseed, u, v);
    ctx.sendMessage(v, last[u] + w);
  }
  bool combine(uint32_t v, uint32_t m) {
    if (m < states[v]) {
      states[v] = m;
      return true;
    }
    return false;
  }
  bool apply(uint32_t v) {
    last[v] = states[v];
    return true;
  }
};

// PageRank_delta (Kernels/PageRank.hpp:129-197): init pr = 0.15, scatter pr/outdeg; combine
// sums; apply adds delta = 0.85 * sum and stays active while delta > 1e-5 (and outdeg > 0),
// scattering delta/outdeg.
struct PageRankDeltaVC : PluginBase {
  typedef double msg_t;
  const OGraph* g;
  std::vector<double> pr, scat, comb;
  bool init(uint32_t v) {
    pr[v] = 0.15;
    if (g->outdeg[v] > 0) {
      scat[v] = pr[v] / (double)g->outdeg[v];
      return true;
    }
    return false;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  bool combine(uint32_t v, double m) {
    comb[v] += m;
    return true;
  }
  bool apply(uint32_t v) {
    const double delta = (1.0 - 0.15) * comb[v];
    pr[v] += delta;
    comb[v] = 0.0;
    if (delta > 1e-5 && g->outdeg[v] > 0) {
      scat[v] = delta / (double)g->outdeg[v];
      return true;
    }
    return false;
  }
};

// SSSP with predecessors (Kernels/SSSP1.hpp:62-95): a message carries (sender, distance); a
// strictly shorter distance replaces both fields.
struct SSSP1VC : PluginBase {
  typedef std::pair<uint32_t, uint32_t> msg_t;  // (pred, dist)
  std::vector<uint32_t> dist, last;
  std::vector<uint64_t> pred;
  uint64_t wseed;
  const uint32_t* warc;
  bool init(uint32_t v) {
    pred[v] = v;
    dist[v] = 0;
    last[v] = 0;
    return true;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t arc) {
    const uint32_t w = warc ? warc[arc] : gre_oracle::sssp_weight(wseed, u, v);
    ctx.sendMessage(v, msg_t(u, last[u] + w));
  }
  bool combine(uint32_t v, const msg_t& m) {
    if (m.second < dist[v]) {
      dist[v] = m.second;
      pred[v] = m.first;
      return true;
    }
    return false;
  }
  bool apply(uint32_t v) {
    last[v] = dist[v];
    return true;
  }
};

// CountIn (Kernels/CountIn.hpp:33-56): every vertex sends 1; apply stores the count received.
struct CountInVC : PluginBase {
  typedef int32_t msg_t;
  std::vector<int32_t> cn, scat, comb;
  bool init(uint32_t v) {
    cn[v] = 0;
    scat[v] = 1;
    return true;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  bool combine(uint32_t v, int32_t m) {
    comb[v] += m;
    return true;
  }
  bool apply(uint32_t v) {
    cn[v] = comb[v];
    return false;
  }
};

// ConnectedComponents (Kernels/CC.hpp:33-67): min global vid label propagation.
struct CCVC : PluginBase {
  typedef uint64_t msg_t;
  std::vector<uint64_t> cc, scat, comb;
  bool init(uint32_t v) {
    cc[v] = v;
    scat[v] = v;
    comb[v] = v;
    return true;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  bool combine(uint32_t v, uint64_t m) {
    if (comb[v] > m) {
      comb[v] = m;
      return true;
    }
    return false;
  }
  bool apply(uint32_t v) {
    if (comb[v] >= cc[v]) return false;
    cc[v] = comb[v];
    scat[v] = cc[v];
    return true;
  }
};

// BC forward (Kernels/BC.hpp:56-91).  numPaths is int in the reference; here it is a double
// (exact below 2^53) and `overflow` records whether an int32 would have wrapped.
struct ForwardVC : PluginBase {
  typedef double msg_t;
  std::vector<int32_t>* level;
  std::vector<double>* sigma;
  std::vector<double> scat, sum;
  int currLevel = 1;
  bool overflow = false;
  bool init(uint32_t v) {
    (*sigma)[v] = 1;
    (*level)[v] = 0;
    scat[v] = 1;
    return true;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, scat[u]); }
  bool combine(uint32_t v, double m) {
    sum[v] += m;
    return true;
  }
  bool apply(uint32_t v) {
    if ((*level)[v] < 0) {
      (*level)[v] = currLevel;
      (*sigma)[v] = sum[v];
      if (sum[v] > 2147483647.0) overflow = true;
      scat[v] = sum[v];
      return true;
    }
    return false;
  }
  void reduce() { currLevel++; }
};

// BC backward (Kernels/BC.hpp:132-163): one superstep per level, `sum` is never reset between
// levels (safe because BFS levels differ by at most one across an arc).
struct BackwardVC : PluginBase {
  typedef double msg_t;
  const std::vector<int32_t>* level;
  const std::vector<double>* sigma;
  std::vector<double>* dep;
  std::vector<double> pathwgt, sum;
  int currLevel = 0;
  bool init(uint32_t v) {
    if ((*level)[v] == currLevel) {
      pathwgt[v] = (1.0 + (*dep)[v]) / (*sigma)[v];
      return true;
    }
    return false;
  }
  template <class C>
  void scatter(C& ctx, uint32_t u, uint32_t v, uint64_t) { ctx.sendMessage(v, pathwgt[u]); }
  bool combine(uint32_t v, double m) {
    sum[v] += m;
    return true;
  }
  bool apply(uint32_t v) {
    if ((*level)[v] == currLevel - 1) (*dep)[v] = sum[v] * (*sigma)[v];
    return false;
  }
};

void copy_trace(const Trace& tr, uint64_t* counts, uint32_t cap, uint32_t* nss) {
  if (nss) *nss = tr.supersteps;
  if (counts)
    for (uint32_t i = 0; i < cap && i < tr.active.size(); ++i) counts[i] = tr.active[i];
}

// One source of Brandes' algorithm exactly as usr/test_bc.cpp:63-110 drives it.
void bc_one_source(const OGraph& g, uint32_t s, std::vector<int32_t>& level, std::vector<double>& sigma,
                   std::vector<double>& dep, bool* overflow) {
  const uint64_t n = g.n;
  level.assign(n, -1);
  sigma.assign(n, 0.0);
  dep.assign(n, 0.0);
  ForwardVC f;
  f.level = &level;
  f.sigma = &sigma;
  f.scat.assign(n, 0.0);
  f.sum.assign(n, 0.0);
  run(g, f, DIR_OUT, &s, 1, 1024, nullptr);
  if (f.overflow && overflow) *overflow = true;
  const int nLevels = f.currLevel;
  BackwardVC b;
  b.level = &level;
  b.sigma = &sigma;
  b.dep = &dep;
  b.pathwgt.assign(n, 0.0);
  b.sum.assign(n, 0.0);
  for (int i = nLevels - 2; i >= 0; --i) {
    b.currLevel = i;
    run(g, b, DIR_IN, nullptr, 0, 1024, nullptr);
  }
}

}  // namespace

// ==============================================================================================
// C ABI used by the tests (ctypes).
// ==============================================================================================
extern "C" {

typedef struct OGraph oracle_graph;

// Loader restated from GraphIngress::loadMetaFromFile / loadEdgesFromFiles at np = 1.
int oracle_load(const char* prefix, oracle_graph** out) {
  std::string meta = std::string(prefix) + ".meta";
  FILE* f = fopen(meta.c_str(), "r");
  if (!f) return 10;
  unsigned long long nv = 0, ne = 0;
  if (fscanf(f, "%llu %llu", &nv, &ne) != 2) {
    fclose(f);
    return 10;
  }
  fclose(f);
  std::vector<uint32_t> src, dst;
  for (int i = 0;; ++i) {
    std::string name = std::string(prefix) + ".edges." + std::to_string(i);
    FILE* e = fopen(name.c_str(), "r");
    if (!e) break;
    char line[256];
    while (fgets(line, sizeof line, e)) {
      if (line[0] == '\n' || line[0] == '\r' || line[0] == '#' || line[0] == 0) continue;
      char* t;
      unsigned long u = strtoul(line, &t, 10);
      unsigned long v = strtoul(t, nullptr, 10);
      if (u >= nv || v >= nv) {
        fclose(e);
        return 9;
      }
      src.push_back((uint32_t)u);
      dst.push_back((uint32_t)v);
    }
    fclose(e);
  }
  OGraph* g = new OGraph;
  g->n = nv;
  build(g, src, dst);
  *out = g;
  return 0;
}

// CSR given directly (source-major); the reverse CSR is built as rbuild does.
int oracle_from_csr(uint64_t n, uint64_t m, const uint64_t* off, const uint32_t* col, oracle_graph** out) {
  std::vector<uint32_t> src(m), dst(m);
  for (uint64_t u = 0; u < n; ++u)
    for (uint64_t a = off[u]; a < off[u + 1]; ++a) {
      src[a] = (uint32_t)u;
      dst[a] = col[a];
    }
  OGraph* g = new OGraph;
  g->n = n;
  build(g, src, dst);
  *out = g;
  return 0;
}

void oracle_free(oracle_graph* g) { delete g; }
uint64_t oracle_num_vertices(const oracle_graph* g) { return g->n; }
uint64_t oracle_num_arcs(const oracle_graph* g) { return g->m; }
void oracle_csr(const oracle_graph* g, uint64_t* off, uint32_t* col) {
  memcpy(off, g->off.data(), sizeof(uint64_t) * (g->n + 1));
  memcpy(col, g->col.data(), sizeof(uint32_t) * g->m);
}

// PageRank on the engine: variant 0 = reference PageRank, 1 = PageRankIter.
// teleport may be null (1-d everywhere).
int oracle_pagerank(const oracle_graph* g, int variant, double d, const double* teleport, uint32_t supersteps,
                    double* pr, uint64_t* counts, uint32_t cap, uint32_t* nss) {
  PageRankVC vc;
  vc.g = g;
  vc.d = d;
  vc.teleport = teleport;
  vc.refresh = variant != 0;
  vc.pr.assign(g->n, 0.0);
  vc.scat.assign(g->n, 0.0);
  vc.comb.assign(g->n, 0.0);
  Trace tr;
  run(*g, vc, DIR_OUT, nullptr, 0, supersteps, &tr);
  memcpy(pr, vc.pr.data(), sizeof(double) * g->n);
  copy_trace(tr, counts, cap, nss);
  return 0;
}

// Personalised PageRank for k one-hot restart vectors (seed vertices), one engine run each:
// out[i*n + v] = x_i(v), x_i = (1-d)·e_seed + d·A^T D^-1 x_i.
int oracle_ppr(const oracle_graph* g, const uint32_t* seeds, uint32_t k, double d, uint32_t supersteps,
               double* out) {
  const uint64_t n = g->n;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < (int64_t)k; ++i) {
    std::vector<double> tele(n, 0.0);
    tele[seeds[i]] = 1.0 - d;
    PageRankVC vc;
    vc.g = g;
    vc.d = d;
    vc.teleport = tele.data();
    vc.refresh = true;
    vc.pr.assign(n, 0.0);
    vc.scat.assign(n, 0.0);
    vc.comb.assign(n, 0.0);
    run(*g, vc, DIR_OUT, nullptr, 0, supersteps, nullptr);
    memcpy(out + (uint64_t)i * n, vc.pr.data(), sizeof(double) * n);
  }
  return 0;
}

// BFS plugin, run<dir> from one source; level[v] = depth in the pred tree, -1 if unreached.
int oracle_bfs(const oracle_graph* g, uint32_t src, int dir, int32_t* level, uint64_t* pred,
               uint64_t* counts, uint32_t cap, uint32_t* nss) {
  BFSVC vc;
  vc.pred.assign(g->n, ~0ull);
  vc.scat.assign(g->n, 0);
  vc.comb.assign(g->n, ~0ull);
  vc.level.assign(g->n, -1);
  Trace tr;
  run(*g, vc, dir, &src, 1, 1024, &tr);
  memcpy(level, vc.level.data(), sizeof(int32_t) * g->n);
  if (pred) memcpy(pred, vc.pred.data(), sizeof(uint64_t) * g->n);
  copy_trace(tr, counts, cap, nss);
  return 0;
}

// Many sources, one independent run each (levels[i*n + v]).
int oracle_bfs_many(const oracle_graph* g, const uint32_t* srcs, uint32_t k, int dir, int32_t* levels) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < (int64_t)k; ++i)
    oracle_bfs(g, srcs[i], dir, levels + (uint64_t)i * g->n, nullptr, nullptr, 0, nullptr);
  return 0;
}

// SSSP plugin, run<Out> (the test_sssp driver's default) from one source.  warc (forward-arc
// order) overrides the harness weight function when non-null.
int oracle_sssp(const oracle_graph* g, uint32_t src, uint64_t wseed, const uint32_t* warc, uint32_t* dist,
                uint64_t* counts, uint32_t cap, uint32_t* nss) {
  SSSPVC vc;
  vc.states.assign(g->n, 0xffffffffu);
  vc.last.assign(g->n, 0);
  vc.wseed = wseed;
  vc.warc = warc;
  Trace tr;
  run(*g, vc, DIR_OUT, &src, 1, 1024, &tr);
  memcpy(dist, vc.states.data(), sizeof(uint32_t) * g->n);
  copy_trace(tr, counts, cap, nss);
  return 0;
}

int oracle_sssp_many(const oracle_graph* g, const uint32_t* srcs, uint32_t k, uint64_t wseed,
                     const uint32_t* warc, uint32_t* dist) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < (int64_t)k; ++i)
    oracle_sssp(g, srcs[i], wseed, warc, dist + (uint64_t)i * g->n, nullptr, 0, nullptr);
  return 0;
}

// PageRank_delta, run<Out> from every vertex (usr/test_pagerank.cpp:65-74 with the
// PageRank_delta typedef of line 22).
int oracle_pagerank_delta(const oracle_graph* g, uint32_t max_ss, double* pr, uint64_t* counts, uint32_t cap, uint32_t* nss) {
  PageRankDeltaVC vc;
  vc.g = g;
  vc.pr.assign(g->n, 0.0);
  vc.scat.assign(g->n, 0.0);
  vc.comb.assign(g->n, 0.0);
  Trace tr;
  run(*g, vc, DIR_OUT, nullptr, 0, max_ss, &tr);
  memcpy(pr, vc.pr.data(), sizeof(double) * g->n);
  copy_trace(tr, counts, cap, nss);
  return 0;
}

// SSSP1 from one source, run<Out> (usr/test_sssp.cpp:58-69 with the SSSP1 include).
int oracle_sssp1(const oracle_graph* g, uint32_t src, uint64_t wseed, const uint32_t* warc, uint32_t* dist, uint64_t* pred,
                 uint64_t* counts, uint32_t cap, uint32_t* nss) {
  SSSP1VC vc;
  vc.dist.assign(g->n, 0xffffffffu);  // _Data(): dist max, pred -1
  vc.pred.assign(g->n, ~0ull);
  vc.last.assign(g->n, 0xffffffffu);
  vc.wseed = wseed;
  vc.warc = warc;
  Trace tr;
  run(*g, vc, DIR_OUT, &src, 1, 1024, &tr);
  memcpy(dist, vc.dist.data(), sizeof(uint32_t) * g->n);
  memcpy(pred, vc.pred.data(), sizeof(uint64_t) * g->n);
  copy_trace(tr, counts, cap, nss);
  return 0;
}

// CountIn with every vertex active along `dir` for max_ss supersteps (usr/test_cIn.cpp:30-40:
// run<In>, one superstep).
int oracle_count_in(const oracle_graph* g, int dir, uint32_t max_ss, int32_t* cn, uint64_t* counts, uint32_t cap,
                    uint32_t* nss) {
  CountInVC vc;
  vc.cn.assign(g->n, 0);
  vc.scat.assign(g->n, 0);
  vc.comb.assign(g->n, 0);
  Trace tr;
  run(*g, vc, dir, nullptr, 0, max_ss, &tr);
  memcpy(cn, vc.cn.data(), sizeof(int32_t) * g->n);
  copy_trace(tr, counts, cap, nss);
  return 0;
}

// ConnectedComponents, run<InOut> with every vertex active (usr/test_cc.cpp:49-60).
int oracle_cc(const oracle_graph* g, uint64_t* label, uint64_t* counts, uint32_t cap, uint32_t* nss) {
  CCVC vc;
  vc.cc.assign(g->n, ~0ull);
  vc.scat.assign(g->n, 0);
  vc.comb.assign(g->n, ~0ull);
  Trace tr;
  run(*g, vc, DIR_INOUT, nullptr, 0, 1024, &tr);
  memcpy(label, vc.cc.data(), sizeof(uint64_t) * g->n);
  copy_trace(tr, counts, cap, nss);
  return 0;
}

// Betweenness: bc[v] = sum over sources s != v of the reference's dependency dep_s(v).
// Also returns, when non-null, the last source's level / sigma / dependency arrays.
// Returns 1 in *overflow when an int32 numPaths would have wrapped for some source.
int oracle_bc(const oracle_graph* g, const uint32_t* srcs, uint32_t k, double* bc, int* overflow,
              double* per_source_dep) {
  const uint64_t n = g->n;
  std::vector<std::vector<double>> deps(k);
  int ovf = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : ovf)
  for (int64_t i = 0; i < (int64_t)k; ++i) {
    std::vector<int32_t> level;
    std::vector<double> sigma;
    bool o = false;
    bc_one_source(*g, srcs[i], level, sigma, deps[i], &o);
    if (o) ovf = 1;
  }
  for (uint64_t v = 0; v < n; ++v) bc[v] = 0.0;
  for (uint32_t i = 0; i < k; ++i) {  // accumulate in source order
    for (uint64_t v = 0; v < n; ++v)
      if (v != srcs[i]) bc[v] += deps[i][v];
    if (per_source_dep) memcpy(per_source_dep + (uint64_t)i * n, deps[i].data(), sizeof(double) * n);
  }
  if (overflow) *overflow = ovf;
  return 0;
}

// BC forward state of one source (levels and path counts), for kernel-level checks.
int oracle_bc_forward(const oracle_graph* g, uint32_t s, int32_t* level, double* sigma, double* dep) {
  std::vector<int32_t> l;
  std::vector<double> sg, dp;
  bool o = false;
  bc_one_source(*g, s, l, sg, dp, &o);
  memcpy(level, l.data(), sizeof(int32_t) * g->n);
  memcpy(sigma, sg.data(), sizeof(double) * g->n);
  if (dep) memcpy(dep, dp.data(), sizeof(double) * g->n);
  return o ? 1 : 0;
}

// Weighted PageRank (no reference counterpart; FP64 Jacobi iteration):
//   s_u = sum_k W_uk, P = D_s^-1 W (dangling rows zero), r = (1-d)·pers + d·P^T r,
// W given per forward arc; `iters` Jacobi steps from r0 = (1-d)·pers.
int oracle_pagerank_weighted(const oracle_graph* g, const double* warc, const double* pers, double d,
                             uint32_t iters, double* r) {
  const uint64_t n = g->n;
  std::vector<double> s(n, 0.0), x(n), y(n);
  for (uint64_t u = 0; u < n; ++u)
    for (uint64_t a = g->off[u]; a < g->off[u + 1]; ++a) s[u] += warc[a];
  for (uint64_t v = 0; v < n; ++v) x[v] = (1.0 - d) * pers[v];
  for (uint32_t it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
      double acc = 0.0;
      for (uint64_t a = g->roff[v]; a < g->roff[v + 1]; ++a) {
        const uint32_t u = g->rcol[a];
        acc += warc[g->rarc[a]] / s[u] * x[u];
      }
      y[v] = (1.0 - d) * pers[v] + d * acc;
    }
    x.swap(y);
  }
  memcpy(r, x.data(), sizeof(double) * n);
  return 0;
}

// Adjoint of the weighted PageRank above for L = c^T r:
//   lambda = c + d·P·lambda, dL/dpers = (1-d)·lambda,
//   dL/dW_uv = d·r_u/s_u·(lambda_v - sum_k P_uk lambda_k)   (forward-arc order).
int oracle_pagerank_adjoint(const oracle_graph* g, const double* warc, const double* r, const double* c,
                            double d, uint32_t iters, double* lambda, double* grad_pers, double* grad_w) {
  const uint64_t n = g->n;
  std::vector<double> s(n, 0.0), x(n), y(n);
  for (uint64_t u = 0; u < n; ++u)
    for (uint64_t a = g->off[u]; a < g->off[u + 1]; ++a) s[u] += warc[a];
  for (uint64_t v = 0; v < n; ++v) x[v] = c[v];
  for (uint32_t it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
      double acc = 0.0;
      for (uint64_t a = g->off[u]; a < g->off[u + 1]; ++a) acc += warc[a] / s[u] * x[g->col[a]];
      y[u] = c[u] + d * acc;
    }
    x.swap(y);
  }
  memcpy(lambda, x.data(), sizeof(double) * n);
  for (uint64_t v = 0; v < n; ++v) grad_pers[v] = (1.0 - d) * x[v];
  for (uint64_t u = 0; u < n; ++u) {
    double pl = 0.0;
    for (uint64_t a = g->off[u]; a < g->off[u + 1]; ++a) pl += warc[a] / s[u] * x[g->col[a]];
    for (uint64_t a = g->off[u]; a < g->off[u + 1]; ++a) grad_w[a] = d * r[u] / s[u] * (x[g->col[a]] - pl);
  }
  return 0;
}

uint32_t oracle_sssp_weight(uint64_t wseed, uint32_t u, uint32_t v) { return gre_oracle::sssp_weight(wseed, u, v); }

}  // extern "C"
