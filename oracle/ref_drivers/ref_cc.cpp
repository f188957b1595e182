// ORACLE — test infrastructure only.  Runs the reference ConnectedComponents plugin
// (Kernels/CC.hpp) on the reference engine, np = 1, exactly as usr/test_cc.cpp: ingress<InOut>,
// srcSet.setALL(), engine.run<InOut>.
//
//   ref_cc <prefix> <out.u64> [repeats]
// Writes n uint64 labels (the minimum global vertex id of each component).
#include "ref_harness.hpp"
#define private public
#define protected public
#include "Kernels/CC.hpp"
#undef private
#undef protected

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s prefix out\n", argv[0]);
    return 2;
  }
  GRE::COMM::Underlying comm;
  comm.init(argc, argv);
  GRE::Util::BufferPool pool;
  pool.config(4096, 8192 * 256, true);
  const std::string prefix(argv[1]), out(argv[2]);
  RefGraph_t g;
  load_graph<InOut>(g, comm, pool, prefix);
  const size_t n = g.get_num_masters();
  GRE::Graph::SourceVertexSet srcSet;
  srcSet.setALL();
  const long repeats = argc > 3 ? atol(argv[3]) : 1;  // independent runs, for timing
  for (long rep = 0; rep < repeats; ++rep) {
    ConnectedComponents cc(g);
    GRE::SynchronousEngine<ConnectedComponents> engine(g, comm, pool, cc);
    engine.initialize();
    comm.startTimer();
    engine.run<InOut>(srcSet, GRE::Par_ThreadPool);
    report_run("cc", comm.stopTimer(), engine.getSuperstepCount());
    write_array(out, cc.cc, sizeof(vid_t) * n);
    engine.finalize();
  }
  comm.finalize();
  pool.finalize();
  return 0;
}
