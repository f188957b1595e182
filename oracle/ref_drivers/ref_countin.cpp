// ORACLE — test infrastructure only.  Runs CountIn (Kernels/CountIn.hpp) on the reference
// engine, np = 1, as usr/test_cIn.cpp: ingress<InOut>, srcSet.setALL(), configMaxSupersteps(1),
// engine.run<In>.
//
//   ref_countin <prefix> <out.i32>
// Writes n int32 counts.
#include "ref_harness.hpp"
#define private public
#define protected public
#include "Kernels/CountIn.hpp"
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
  CountIn countIn(g);
  GRE::SynchronousEngine<CountIn> engine(g, comm, pool, countIn);
  engine.initialize();
  engine.configMaxSupersteps(1);
  comm.startTimer();
  engine.run<In>(srcSet, GRE::Par_ThreadPool);
  report_run("countin", comm.stopTimer(), engine.getSuperstepCount());
  write_array(out, countIn.cn, sizeof(int) * n);
  engine.finalize();
  comm.finalize();
  pool.finalize();
  return 0;
}
