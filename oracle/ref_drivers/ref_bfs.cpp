// ORACLE — test infrastructure only.  For each root of <prefix>.roots, np = 1:
//   1. the reference BFS plugin (Kernels/BFS.hpp) exactly as usr/test_bfs.cpp runs it:
//      ingress<InOut>, srcSet.addVertex(root), engine.run<In>;
//   2. the reference BC Forward plugin (Kernels/BC.hpp:22-95) with run<Out> from the same root,
//      whose `level` field is the BFS level.
// The BFS plugin stores in pred the value it received, and it forwards pred_scatter = pred
// (BFS.hpp:66-72), so every reached vertex ends with pred == root: it marks reachability, not a
// parent tree.  Levels therefore come from Forward; the driver checks that the two runs agree
// on the reached set and prints GRE_BFS_REACH_MISMATCH if they do not.
//
//   ref_bfs <prefix> <out.i32> [max_roots]
// Writes, per root, n int32 levels (-1 = unreached).
#include "ref_harness.hpp"
#define private public
#define protected public
#include "Kernels/BFS.hpp"
#undef private
#undef protected

// BC.hpp declares its own plugin types without the global typedefs of BFS.hpp
#define private public
#define protected public
#include "Kernels/BC.hpp"
#undef private
#undef protected

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s prefix out [max_roots]\n", argv[0]);
    return 2;
  }
  GRE::COMM::Underlying comm;
  comm.init(argc, argv);
  GRE::Util::BufferPool pool;
  pool.config(4096, 8192 * 256, true);
  const std::string prefix(argv[1]), out(argv[2]);
  RefGraph_t g;
  load_graph<InOut>(g, comm, pool, prefix);
  std::vector<vid_t> roots = load_roots(prefix);
  if (argc > 3 && (size_t)atol(argv[3]) < roots.size()) roots.resize((size_t)atol(argv[3]));
  const size_t n = g.get_num_masters();
  write_array(out, "", 0);
  bool mismatch = false;
  for (size_t r = 0; r < roots.size(); ++r) {
    GRE::Graph::SourceVertexSet srcSet;
    srcSet.addVertex(roots[r], g);
    BFS bfs(g);
    GRE::SynchronousEngine<BFS> engine(g, comm, pool, bfs);
    engine.initialize();
    comm.startTimer();
    engine.run<In>(srcSet, GRE::Par_ThreadPool);
    report_run("bfs", comm.stopTimer(), engine.getSuperstepCount());

    vtxData* state = NULL;
    Forward fw(g, state);
    GRE::SynchronousEngine<Forward> fengine(g, comm, pool, fw);
    fengine.initialize();
    comm.startTimer();
    fengine.run<Out>(srcSet, GRE::Par_ThreadPool);
    report_run("bfs_levels", comm.stopTimer(), fengine.getSuperstepCount());
    std::vector<int> level(n, -1);
    for (size_t v = 0; v < n; ++v) {
      level[v] = state[v].level;
      const bool reached_bfs = bfs.pred[v] != (vid_t)-1;
      if (reached_bfs != (level[v] >= 0)) mismatch = true;
      if (reached_bfs && bfs.pred[v] != roots[r]) mismatch = true;
    }
    append_array(out, level.data(), sizeof(int) * n);
    fengine.finalize();
    delete[] state;
    engine.finalize();
  }
  if (mismatch) printf("GRE_BFS_REACH_MISMATCH\n");
  comm.finalize();
  pool.finalize();
  return 0;
}
