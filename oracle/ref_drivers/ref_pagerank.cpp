// ORACLE — test infrastructure only.  Runs the reference PageRank plugin (or the harness
// PageRankIter / personalised plugins written against the reference's VertexCode API) on the
// reference engine, np = 1.
//
//   ref_pagerank <prefix> <out.f64> gre|iter|delta <supersteps> [repeats]
//   ref_pagerank <prefix> <out.f64> ppr <supersteps> <seed vertex> [<seed vertex> ...]
// Writes n doubles per run (appended in seed order for ppr).  Mirrors usr/test_pagerank.cpp:
// ingress<Out>, srcSet.setALL(), configMaxSupersteps, engine.run (= run<Out>).
#include "ref_harness.hpp"
#define private public
#define protected public
#include "Kernels/PageRank.hpp"
#undef private
#undef protected

// PageRank with the scatter value refreshed in apply: the power iteration
// x <- 0.15·w + 0.85·A^T D^-1 x whose first step the reference PageRank repeats
// (Kernels/PageRank.hpp:70-74 never updates pr_scatter).  teleport[v] = 0.15·w_v.
class PageRankIter : public PageRank_Base {
 public:
  PageRankIter(DistributedGraph_t& dg, const std::vector<double>* tele)
      : PageRank_Base(dg), teleport(tele), pr(NULL), pr_combine(NULL), pr_scatter(NULL) {}
  void alloc() {
    allocScatterData(pr_scatter);
    allocCombineData(pr_combine, 0.0);
    allocVertexData(pr);
  }
  void free() {
    freeScatterData(pr_scatter);
    freeCombineData(pr_combine);
    freeVertexData(pr);
  }
  double tele(const lvid_t lv) const { return teleport ? (*teleport)[lv] : 0.15; }
  inline bool init(const lvid_t lv) {
    pr[lv] = tele(lv);
    if (graph.getOutdegree(lv) > 0) {
      pr_scatter[lv] = pr[lv] / (double)graph.getOutdegree(lv);
      return true;
    }
    return false;
  }
  template <typename Ctx_t, typename EdgeIterator_t>
  inline void scatter(Ctx_t& ctx, const lvid_t lsrc, const lvid_t ldst, const EdgeIterator_t& it) {
    ctx.engine->sendMessage(ctx, ldst, pr_scatter[lsrc]);
  }
  template <typename Lock_t>
  inline bool combine(const lvid_t ldst, const combine_data_t& msg, Lock_t& lock) {
    lock.spinLock();
    pr_combine[ldst] += msg;
    lock.unLock();
    return true;
  }
  inline bool apply(const lvid_t lv) {
    pr[lv] = tele(lv) + 0.85 * pr_combine[lv];
    pr_combine[lv] = 0.0;
    if (graph.getOutdegree(lv) > 0) pr_scatter[lv] = pr[lv] / (double)graph.getOutdegree(lv);
    return false;
  }
  inline bool assert_to_halt(const lvid_t lv) { return false; }
  inline void reset_combiner(const lvid_t ldst) { pr_combine[ldst] = 0.0; }

  const std::vector<double>* teleport;
  vertex_data_t* pr;
  combine_data_t* pr_combine;
  scatter_data_t* pr_scatter;
};

int main(int argc, char** argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s prefix out gre|iter|ppr supersteps [seeds...]\n", argv[0]);
    return 2;
  }
  GRE::COMM::Underlying comm;
  comm.init(argc, argv);
  GRE::Util::BufferPool pool;
  pool.config(2048, 8192 * 256, true);
  const std::string prefix(argv[1]), out(argv[2]), variant(argv[3]);
  const long supersteps = atol(argv[4]);
  RefGraph_t g;
  load_graph<Out>(g, comm, pool, prefix);
  const size_t n = g.get_num_masters();
  GRE::Graph::SourceVertexSet srcSet;
  srcSet.setALL();
  // gre / iter: optional argv[5] = number of independent runs (one engine each), for timing
  const long repeats = (variant != "ppr" && argc > 5) ? atol(argv[5]) : 1;
  if (variant == "gre") {
    for (long rep = 0; rep < repeats; ++rep) {
      PageRank pr(g);
      GRE::SynchronousEngine<PageRank> engine(g, comm, pool, pr);
      engine.initialize();
      engine.configMaxSupersteps(supersteps);
      comm.startTimer();
      engine.run(srcSet, GRE::Par_ThreadPool);
      report_run("pagerank", comm.stopTimer(), engine.getSuperstepCount());
      write_array(out, pr.pr, sizeof(double) * n);
      engine.finalize();
    }
  } else if (variant == "iter") {
    for (long rep = 0; rep < repeats; ++rep) {
      PageRankIter pr(g, NULL);
      GRE::SynchronousEngine<PageRankIter> engine(g, comm, pool, pr);
      engine.initialize();
      engine.configMaxSupersteps(supersteps);
      comm.startTimer();
      engine.run(srcSet, GRE::Par_ThreadPool);
      report_run("pagerank_iter", comm.stopTimer(), engine.getSuperstepCount());
      write_array(out, pr.pr, sizeof(double) * n);
      engine.finalize();
    }
  } else if (variant == "delta") {  // the PageRank_delta typedef of usr/test_pagerank.cpp:22
    PageRank_delta pr(g);
    GRE::SynchronousEngine<PageRank_delta> engine(g, comm, pool, pr);
    engine.initialize();
    engine.configMaxSupersteps(supersteps);
    comm.startTimer();
    engine.run(srcSet, GRE::Par_ThreadPool);
    report_run("pagerank_delta", comm.stopTimer(), engine.getSuperstepCount());
    write_array(out, pr.pr, sizeof(double) * n);
    engine.finalize();
  } else if (variant == "ppr") {
    write_array(out, "", 0);
    for (int a = 5; a < argc; ++a) {
      std::vector<double> tele(n, 0.0);
      tele[strtoul(argv[a], NULL, 10)] = 0.15;
      PageRankIter pr(g, &tele);
      GRE::SynchronousEngine<PageRankIter> engine(g, comm, pool, pr);
      engine.initialize();
      engine.configMaxSupersteps(supersteps);
      comm.startTimer();
      engine.run(srcSet, GRE::Par_ThreadPool);
      report_run("ppr", comm.stopTimer(), engine.getSuperstepCount());
      append_array(out, pr.pr, sizeof(double) * n);
      engine.finalize();
    }
  } else {
    fprintf(stderr, "unknown variant %s\n", variant.c_str());
    return 2;
  }
  comm.finalize();
  pool.finalize();
  return 0;
}
