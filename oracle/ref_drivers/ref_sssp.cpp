// ORACLE — test infrastructure only.  Runs SSSP on the reference engine, np = 1, once per root
// of <prefix>.roots, as usr/test_sssp.cpp does for one: ingress (Out), addVertex(root),
// engine.run (= run<Out>).
//
//   ref_sssp <prefix> <out.u32> <weight seed> [max_roots]
// The plugin is the reference SSSP (Kernels/SSSP.hpp:55-89) with one change, the weight: the
// reference draws rand()%65535 per CSR slot and looks it up at position/8
// (DistributedGraph.hpp:219-226, LocalGraph.hpp:173-176), which no other program can
// reproduce.  SSSP_W computes the weight of arc (u, v) from the global ids instead, with the
// same function the GPU side is given.  Init, combine and apply are the reference's.
#include "../oracle_common.hpp"
#include "ref_harness.hpp"
#define private public
#define protected public
#include "Kernels/SSSP.hpp"
#undef private
#undef protected

class SSSP_W : public SSSP_Base {
 public:
  SSSP_W(DistributedGraph_t& dg, uint64_t seed) : SSSP_Base(dg), states(NULL), lastStates(NULL), wseed(seed) {}
  void alloc() {
    allocScatterData(lastStates);
    allocCombineData(states, std::numeric_limits<dist_t>::max());
    allocVertexData(states);
  }
  void free() {
    freeScatterData(lastStates);
    freeCombineData(states);
    freeVertexData(states);
  }
  inline bool init(const lvid_t lv) {
    states[lv] = 0;
    lastStates[lv] = states[lv];
    return true;
  }
  template <typename Ctx_t, typename EdgeIterator_t>
  inline void scatter(Ctx_t& ctx, const lvid_t lsrc, const lvid_t ldst, const EdgeIterator_t& it) {
    const dist_t w = gre_oracle::sssp_weight(wseed, graph.get_vid(lsrc), graph.get_vid(ldst));
    scatter_data_t msg(lastStates[lsrc] + w);
    ctx.engine->sendMessage(ctx, ldst, msg);
  }
  template <typename Lock_t>
  inline bool combine(const lvid_t ldst, const combine_data_t& msg, Lock_t& lock) {
    if (msg < states[ldst]) {
      lock.spinLock();
      if (msg < states[ldst]) {
        states[ldst] = msg;
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
  for (size_t r = 0; r < roots.size(); ++r) {
    GRE::Graph::SourceVertexSet srcSet;
    srcSet.addVertex(roots[r], g);
    SSSP_W sssp(g, wseed);
    GRE::SynchronousEngine<SSSP_W> engine(g, comm, pool, sssp);
    engine.initialize();
    engine.configMaxSupersteps(1024);
    comm.startTimer();
    engine.run(srcSet, GRE::Par_ThreadPool);
    report_run("sssp", comm.stopTimer(), engine.getSuperstepCount());
    append_array(out, sssp.states, sizeof(dist_t) * n);
    engine.finalize();
  }
  comm.finalize();
  pool.finalize();
  return 0;
}
