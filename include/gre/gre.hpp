// gre/gre.hpp — C++ host mirror of the reference GRE driver API over the C ABI (gre_gpu.h).
//
// The reference drivers (usr/test_*.cpp) use:
//   DistributedGraph_t g; g.ingress<InOut>(comm, pool, prefix, format, method);
//   SourceVertexSet srcSet; srcSet.addVertex(v, g) | srcSet.setALL();
//   Plugin p(g); SynchronousEngine<Plugin> engine(g, comm, pool, p);
//   engine.initialize(); engine.configMaxSupersteps(n); engine.run<Dir>(srcSet);
//   engine.getSuperstepCount(); engine.finalize();
// (Graph/DistributedGraph.hpp:153-172, Graph/VertexSet.hpp:286-347, Engine/Engine.hpp:94-202).
// This header keeps those names for the five reference plugins.  The communicator and buffer
// pool disappear for one GPU; errors are reported as gre::Error exceptions carrying the
// status code instead of exit(-1).  Results are read from the plugin objects after run().
// An np > 1 job (one GPU per rank) uses Underlying (the communicator) and PartitionedGraph.
#pragma once
#include <stdint.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "../gre_gpu.h"

namespace gre {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& where)
      : std::runtime_error(where + ": " + gre_status_str(s) + " (" + gre_last_error() + ")"), status(s) {}
};

inline void check(int s, const char* where) {
  if (s != GRE_SUCCESS && s != GRE_UNFINISHED) throw Error(s, where);
}

enum Dir { Out = GRE_DIR_OUT, In = GRE_DIR_IN, InOut = GRE_DIR_INOUT };

// DistributedGraph<GraphInCSR> of one rank: every vertex is a master.
class DistributedGraph {
 public:
  DistributedGraph() = default;
  DistributedGraph(const DistributedGraph&) = delete;
  DistributedGraph& operator=(const DistributedGraph&) = delete;
  ~DistributedGraph() {
    if (g_) gre_graph_free(g_);
  }
  // ingress<dir>(comm, pool, prefix, format, method) (DistributedGraph.hpp:153-172):
  //   method "edgelists": the text files <prefix>.meta + <prefix>.edges.<i>;
  //   method "partition" / "partitions": the saved partitions <prefix>.part.<nparts>.<r> of an
  //   np = nparts run (GraphIngress.hpp:86-96, 1024-1071; the reference sets nparts to its rank
  //   count), merged into this one graph.  Like the reference, partitions hold out-arcs, so
  //   dir In is refused (GraphIngress.hpp:92-95).
  // `symmetric` lets the CSR serve as CSC, `reorder` stores vertices by decreasing degree
  // (invisible to callers).
  template <Dir dir>
  bool ingress(const std::string& prefix, const std::string& format = "ascii", const std::string& method = "edgelists",
               bool symmetric = false, bool reorder = false, int device = 0, uint32_t nparts = 1) {
    const bool parts = method == "partition" || method == "partitions";
    if (format != "ascii" || !(parts || method == "edgelists"))
      throw Error(GRE_NOT_IMPLEMENTED, "ingress: ascii edge lists or saved partitions only");
    if (parts && dir == In) throw Error(GRE_NOT_IMPLEMENTED, "ingress: partitions of In edges are not supported");
    if (g_) gre_graph_free(g_);
    g_ = nullptr;
    uint32_t flags = (uint32_t)dir | (symmetric ? GRE_GRAPH_SYMMETRIC : 0u) | (reorder ? GRE_GRAPH_REORDER : 0u);
    if (parts) check(gre_graph_load_parts(prefix.c_str(), nparts, flags, device, &g_), "gre_graph_load_parts");
    else check(gre_graph_load(prefix.c_str(), flags, device, &g_), "gre_graph_load");
    return true;
  }
  size_t get_num_masters() const { return info().first; }
  size_t get_num_edges() const { return info().second; }
  std::vector<uint32_t> getOutdegrees() const {
    std::vector<uint32_t> d(get_num_masters());
    check(gre_graph_outdegree(g_, d.data()), "gre_graph_outdegree");
    return d;
  }
  // loadEdgeProperty (DistributedGraph.hpp:195-226): weights in the arc order of the CSR
  void loadEdgeProperty(const std::vector<uint32_t>& w) { check(gre_graph_set_weights_u32(g_, w.data()), "set_weights"); }
  void loadEdgePropertyHash(uint64_t wseed) { check(gre_graph_set_weights_hash(g_, wseed), "set_weights_hash"); }
  gre_graph handle() const { return g_; }

 private:
  std::pair<size_t, size_t> info() const {
    uint64_t n = 0, m = 0;
    check(gre_graph_info(g_, &n, &m, nullptr), "gre_graph_info");
    return {n, m};
  }
  gre_graph g_ = nullptr;
};

// SourceVertexSet (Graph/VertexSet.hpp:286-347)
struct SourceVertexSet {
  bool complete = false;
  std::vector<uint32_t> vertices;
  void setALL() { complete = true; }
  bool isALL() const { return complete; }
  void addVertex(uint64_t v, const DistributedGraph&) { vertices.push_back((uint32_t)v); }
  void clear() {
    complete = false;
    vertices.clear();
  }
};

// The reference plugins; each keeps its result arrays after the engine ran.
struct PageRank {
  explicit PageRank(DistributedGraph& g, bool iterate = false) : graph(g), iter(iterate) {}
  DistributedGraph& graph;
  bool iter;  // false: Kernels/PageRank.hpp verbatim; true: power iteration (pr_scatter refreshed)
  std::vector<double> pr;
};
struct BFS {
  explicit BFS(DistributedGraph& g) : graph(g) {}
  DistributedGraph& graph;
  std::vector<uint64_t> pred;  // source vid on reached vertices (the plugin forwards pred)
  std::vector<int32_t> level;
};
struct SSSP {
  explicit SSSP(DistributedGraph& g) : graph(g) {}
  DistributedGraph& graph;
  std::vector<uint32_t> states;  // distances
};
struct ConnectedComponents {
  explicit ConnectedComponents(DistributedGraph& g) : graph(g) {}
  DistributedGraph& graph;
  std::vector<uint32_t> cc;  // minimum vid of the component
};
struct PageRank_delta {  // Kernels/PageRank.hpp:129-197
  explicit PageRank_delta(DistributedGraph& g) : graph(g) {}
  DistributedGraph& graph;
  std::vector<double> pr;
};
struct SSSP1 {  // Kernels/SSSP1.hpp: distances and predecessors
  explicit SSSP1(DistributedGraph& g) : graph(g) {}
  DistributedGraph& graph;
  std::vector<uint32_t> dist;
  std::vector<uint64_t> pred;  // caller vid of the predecessor; UINT64_MAX when unreached
};
struct CountIn {  // Kernels/CountIn.hpp
  explicit CountIn(DistributedGraph& g) : graph(g) {}
  DistributedGraph& graph;
  std::vector<int32_t> cn;
};
struct BC {  // usr/test_bc.cpp's Forward + Backward, accumulated over the sources
  explicit BC(DistributedGraph& g) : graph(g) {}
  DistributedGraph& graph;
  std::vector<double> bc;
};

// SynchronousEngine<VertexCode> (Engine/Engine.hpp:54-1418) for the plugins above.
template <class VC>
class SynchronousEngine {
 public:
  SynchronousEngine(DistributedGraph& g, VC& vc) : g_(g), vc_(vc) {}
  void initialize() {}
  void finalize() {}
  void configMaxSupersteps(long n) { max_ = n > 0 ? (uint32_t)n : 1024; }
  long getSuperstepCount() const { return st_.supersteps; }
  const gre_stats& stats() const { return st_; }
  template <Dir dir = Out>
  void run(const SourceVertexSet& src) {
    runImpl(dir, src, vc_);
  }

 private:
  const uint32_t* first(const SourceVertexSet& s) const {
    if (s.vertices.empty()) throw Error(GRE_INVALID_ARG, "run: no source vertex");
    return s.vertices.data();
  }
  void runImpl(Dir, const SourceVertexSet&, PageRank& p) {
    p.pr.resize(g_.get_num_masters());
    check(gre_vc_pagerank(g_.handle(), p.iter ? GRE_PR_ITER : GRE_PR_REFERENCE, max_, p.pr.data(), &st_), "gre_vc_pagerank");
  }
  void runImpl(Dir dir, const SourceVertexSet& s, BFS& b) {
    b.pred.resize(g_.get_num_masters());
    b.level.resize(g_.get_num_masters());
    check(gre_vc_bfs(g_.handle(), *first(s), (int)dir, b.pred.data(), b.level.data(), &st_), "gre_vc_bfs");
  }
  void runImpl(Dir, const SourceVertexSet& s, SSSP& p) {
    p.states.resize(g_.get_num_masters());
    check(gre_vc_sssp(g_.handle(), *first(s), max_, p.states.data(), &st_), "gre_vc_sssp");
  }
  void runImpl(Dir, const SourceVertexSet&, PageRank_delta& p) {
    p.pr.resize(g_.get_num_masters());
    check(gre_vc_pagerank_delta(g_.handle(), max_, p.pr.data(), &st_), "gre_vc_pagerank_delta");
  }
  void runImpl(Dir, const SourceVertexSet& s, SSSP1& p) {
    p.dist.resize(g_.get_num_masters());
    p.pred.resize(g_.get_num_masters());
    check(gre_vc_sssp1(g_.handle(), *first(s), max_, p.dist.data(), p.pred.data(), &st_), "gre_vc_sssp1");
  }
  void runImpl(Dir dir, const SourceVertexSet&, CountIn& c) {
    c.cn.resize(g_.get_num_masters());
    check(gre_vc_count_in(g_.handle(), (int)dir, max_, c.cn.data(), &st_), "gre_vc_count_in");
  }
  void runImpl(Dir, const SourceVertexSet&, ConnectedComponents& c) {
    c.cc.resize(g_.get_num_masters());
    check(gre_vc_cc(g_.handle(), c.cc.data(), &st_), "gre_vc_cc");
  }
  void runImpl(Dir, const SourceVertexSet& s, BC& b) {
    b.bc.resize(g_.get_num_masters());
    check(gre_vc_bc(g_.handle(), s.vertices.data(), (uint32_t)s.vertices.size(), b.bc.data(), &st_), "gre_vc_bc");
  }

  DistributedGraph& g_;
  VC& vc_;
  uint32_t max_ = 1024;
  gre_stats st_{};
};

// Graph::EdgePartition (Graph/GraphIngress.hpp:1272-1452): the offline partitioner, driven as
// usr/debug/test_graphPar.cpp drives it (`EdgePartition par; par.divideEdges(prefix, n);`).  It
// writes <prefix>.part.<n>.<r>, .outdegree.<n>.<p> and .scatterMap.<n>.<p> from the edge lists,
// on the host (gre_partition_edges); errors throw gre::Error instead of printing.
class EdgePartition {
 public:
  void divideEdges(const std::string& prefix, const int n) {
    counts_.assign(n > 0 ? n : 1, 0);
    check(gre_partition_edges(prefix.c_str(), n > 0 ? (uint32_t)n : 0u, counts_.data()), "gre_partition_edges");
    counts_.resize(n > 0 ? n : 0);
  }
  const std::vector<uint64_t>& partEdges() const { return counts_; }  // edges per part of the last split

 private:
  std::vector<uint64_t> counts_;
};

// COMM::Underlying (Comm/CommUnderlying.hpp:25-80) of an np > 1 job: the library's NCCL
// communicator over the job's ranks, rank() and size() as in the reference.  Agreeing on the
// ranks (MPI_Init's part) is the job's: rank 0 makes the id with uniqueId() and hands it to every
// rank (a file, a launcher, a socket); each rank builds its communicator on its device.
class Underlying {
 public:
  static std::vector<uint8_t> uniqueId() {
    std::vector<uint8_t> id(128);
    check(gre_nccl_unique_id(id.data()), "gre_nccl_unique_id");
    return id;
  }
  Underlying(const std::vector<uint8_t>& id, int size, int rank, int device = 0) : size_(size), rank_(rank) {
    if (id.size() != 128) throw Error(GRE_INVALID_ARG, "Underlying: the id has 128 bytes");
    check(gre_nccl_create(id.data(), (uint32_t)size, (uint32_t)rank, device, &c_), "gre_nccl_create");
  }
  Underlying(const Underlying&) = delete;
  Underlying& operator=(const Underlying&) = delete;
  ~Underlying() {
    if (c_) gre_nccl_free(c_);
  }
  int rank() const { return rank_; }
  int size() const { return size_; }
  gre_nccl handle() const { return c_; }

 private:
  gre_nccl c_ = nullptr;
  int size_ = 1, rank_ = 0;
};

// This rank's part of a graph split by vertex over the ranks of `comm` (gre_part_create):
// built from the graph the rank loaded, which may be released afterwards.  Every rank gets the
// results of all vertices.
class PartitionedGraph {
 public:
  PartitionedGraph(const DistributedGraph& g, Underlying& comm) : comm_(comm), n_(g.get_num_masters()) {
    check(gre_part_create(g.handle(), (uint32_t)comm.size(), (uint32_t)comm.rank(), &p_), "gre_part_create");
  }
  PartitionedGraph(const PartitionedGraph&) = delete;
  PartitionedGraph& operator=(const PartitionedGraph&) = delete;
  ~PartitionedGraph() {
    if (p_) gre_part_free(p_);
  }
  std::vector<int32_t> bfs(uint32_t src, gre_stats* st = nullptr) {
    std::vector<int32_t> level(n_);
    check(gre_part_bfs(p_, src, level.data(), gre_nccl_exchange, comm_.handle(), st), "gre_part_bfs");
    return level;
  }
  std::vector<uint32_t> sssp(uint32_t src, gre_stats* st = nullptr) {
    std::vector<uint32_t> dist(n_);
    check(gre_part_sssp(p_, src, dist.data(), gre_nccl_exchange, comm_.handle(), st), "gre_part_sssp");
    return dist;
  }
  std::vector<uint32_t> cc(gre_stats* st = nullptr) {
    std::vector<uint32_t> label(n_);
    check(gre_part_cc(p_, label.data(), gre_nccl_exchange, comm_.handle(), st), "gre_part_cc");
    return label;
  }
  std::vector<double> pagerank(bool iter, double d, uint32_t iters, gre_stats* st = nullptr) {
    std::vector<double> pr(n_);
    check(gre_part_pagerank(p_, iter ? GRE_PR_ITER : GRE_PR_REFERENCE, d, iters, pr.data(), gre_nccl_exchange,
                            comm_.handle(), st),
          "gre_part_pagerank");
    return pr;
  }

 private:
  Underlying& comm_;
  size_t n_;
  gre_part p_ = nullptr;
};

}  // namespace gre
