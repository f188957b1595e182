// ORACLE — test infrastructure only.  Runs the reference BC plugins (Kernels/BC.hpp Forward and
// Backward) on the reference engine, np = 1, for each root of <prefix>.roots, with the
// two-phase loop of usr/test_bc.cpp:63-110, and accumulates bc(v) = sum_{s != v} dep_s(v)
// (the reference driver handles one source and keeps no total).
//
//   ref_bc <prefix> <out.f64> [max_roots]
// Writes n doubles.  Prints "GRE_BC_OVERFLOW" when some numPaths (int32 in the reference,
// BC.hpp:12-17) is not positive for a reached vertex, i.e. when it wrapped.
#include "ref_harness.hpp"
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
  pool.config(2048, 8192 * 256, true);
  const std::string prefix(argv[1]), out(argv[2]);
  RefGraph_t g;
  load_graph<InOut>(g, comm, pool, prefix);
  std::vector<vid_t> roots = load_roots(prefix);
  if (argc > 3 && (size_t)atol(argv[3]) < roots.size()) roots.resize((size_t)atol(argv[3]));
  const size_t n = g.get_num_masters();
  std::vector<double> bc(n, 0.0);
  bool overflow = false;
  for (size_t r = 0; r < roots.size(); ++r) {
    GRE::Graph::SourceVertexSet srcSet;
    srcSet.addVertex(roots[r], g);
    vtxData* vtxState = NULL;
    Forward bfs(g, vtxState);
    GRE::SynchronousEngine<Forward> fengine(g, comm, pool, bfs);
    fengine.initialize();
    comm.startTimer();
    fengine.run<Out>(srcSet, GRE::Par_ThreadPool);
    const double t1 = comm.stopTimer();
    const int nLevels = bfs.getCurrLevel();
    fengine.finalize();

    double* dependencies = NULL;
    Backward bp(g, vtxState, dependencies);
    GRE::SynchronousEngine<Backward> bengine(g, comm, pool, bp);
    bengine.initialize();
    comm.startTimer();
    for (int i = nLevels - 2; i >= 0; i--) {
      srcSet.setALL();
      bp.setCurrLevel(i);
      bengine.run<In>(srcSet, GRE::Par_ThreadPool);
    }
    const double t2 = comm.stopTimer();
    report_run("bc", t1 + t2, nLevels);
    for (size_t v = 0; v < n; ++v) {
      if (vtxState[v].level >= 0 && vtxState[v].numPaths <= 0) overflow = true;
      if (v != roots[r]) bc[v] += dependencies[v];
    }
    bengine.finalize();
    delete[] vtxState;
    delete[] dependencies;
  }
  if (overflow) printf("GRE_BC_OVERFLOW\n");
  write_array(out, bc.data(), sizeof(double) * n);
  comm.finalize();
  pool.finalize();
  return 0;
}
