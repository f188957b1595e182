// ORACLE — test infrastructure only.  Runs SSSP with predecessors (Kernels/SSSP1.hpp) on the
// reference engine, np = 1, once per root of <prefix>.roots, as usr/test_sssp.cpp does with its
// commented-out SSSP1 include: ingress (Out), addVertex(root), engine.run (= run<Out>).
//
//   ref_sssp1 <prefix> <out.bin> <weight seed> [max_roots]
// Per root writes n uint32 distances then n uint64 predecessors.  The weight is the harness
// weight of the arc's endpoints (see ref_sssp.cpp); init, combine and apply are SSSP1.hpp's.
#include "../oracle_common.hpp"
#include "ref_harness.hpp"
#define private public
#define protected public
#include "Kernels/SSSP1.hpp"
#undef private
#undef protected

class SSSP1_W : public SSSP_Base {
 public:
  SSSP1_W(DistributedGraph_t& dg, uint64_t seed) : SSSP_Base(dg), states(NULL), lastStates(NULL), wseed(seed) {}
  void alloc() {
    allocScatterData(lastStates);
    allocCombineData(states);
    allocVertexData(states);
  }
  void free() {
    freeScatterData(lastStates);
    freeCombineData(states);
    freeVertexData(states);
  }
  inline bool init(const lvid_t lv) {
    states[lv].pred = graph.get_vid(lv);
    states[lv].dist = 0;
    lastStates[lv] = states[lv];
    return true;
  }
  template <typename Ctx_t, typename EdgeIterator_t>
  inline void scatter(Ctx_t& ctx, const lvid_t lsrc, const lvid_t ldst, const EdgeIterator_t& it) {
    const dist_t w = gre_oracle::sssp_weight(wseed, graph.get_vid(lsrc), graph.get_vid(ldst));
    scatter_data_t msg(lsrc, lastStates[lsrc].dist + w);
    ctx.engine->sendMessage(ctx, ldst, msg);
  }
  template <typename Lock_t>
  inline bool combine(const lvid_t ldst, const combine_data_t& msg, Lock_t& lock) {
    if (msg.dist < states[ldst].dist) {
      lock.spinLock();
      if (msg.dist < states[ldst].dist) {
        states[ldst].dist = msg.dist;
        states[ldst].pred = msg.pred;
        lock.unLock();
        return true;
      }
      lock.unLock();
    }
    return false;
  }
  inline bool apply(const lvid_t lv) {
    lastStates[lv] = states[lv];
    return true;
  }
  inline void reset_combiner(const lvid_t ldst) {}
  inline void reset_scatter(const lvid_t lsrc) {}

  vertex_data_t* states;
  scatter_data_t* lastStates;
  uint64_t wseed;
};

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s prefix out wseed [max_roots]\n", argv[0]);
    return 2;
  }
  GRE::COMM::Underlying comm;
  comm.init(argc, argv);
  GRE::Util::BufferPool pool;
  pool.config(4096, 8192 * 256, true);
  const std::string prefix(argv[1]), out(argv[2]);
  const uint64_t wseed = strtoull(argv[3], NULL, 10);
  RefGraph_t g;
  load_graph<Out>(g, comm, pool, prefix);
  std::vector<vid_t> roots = load_roots(prefix);
  if (argc > 4 && (size_t)atol(argv[4]) < roots.size()) roots.resize((size_t)atol(argv[4]));
  const size_t n = g.get_num_masters();
  write_array(out, "", 0);
  std::vector<uint32_t> dist(n);
  std::vector<uint64_t> pred(n);
  for (size_t r = 0; r < roots.size(); ++r) {
    GRE::Graph::SourceVertexSet srcSet;
    srcSet.addVertex(roots[r], g);
    SSSP1_W sssp(g, wseed);
    GRE::SynchronousEngine<SSSP1_W> engine(g, comm, pool, sssp);
    engine.initialize();
    engine.configMaxSupersteps(1024);
    comm.startTimer();
    engine.run(srcSet, GRE::Par_ThreadPool);
    report_run("sssp1", comm.stopTimer(), engine.getSuperstepCount());
    for (size_t v = 0; v < n; ++v) {
      dist[v] = sssp.states[v].dist;
      pred[v] = sssp.states[v].pred;
    }
    append_array(out, dist.data(), sizeof(uint32_t) * n);
    append_array(out, pred.data(), sizeof(uint64_t) * n);
    engine.finalize();
  }
  comm.finalize();
  pool.finalize();
  return 0;
}
