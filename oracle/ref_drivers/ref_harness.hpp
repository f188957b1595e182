// ORACLE — test infrastructure only.  Shared driver code for running the reference GRE engine
// (compiled from its own headers) on this project's inputs.
//
// Mirrors the reference drivers (usr/test_*.cpp): ingress, one SynchronousEngine per run,
// MPI_Wtime around engine.run only (usr/test_bfs.cpp:67-71).  Two deviations, both forced by the
// toolchain and neither touching the engine or plugins:
//   * DistributedGraph::ingress<dir>(comm, pool, params) lacks the `template` keyword on a
//     dependent call (Graph/DistributedGraph.hpp:165) and does not compile; load_graph() below
//     performs the same three steps (DistributedGraph.hpp:161-172) by calling the reference's
//     GraphIngress directly;
//   * the build passes -fno-unreachable-traps so that the reference's non-void functions that
//     end without `return` (Engine.hpp:207-223, GraphIngress.hpp:76-304) return instead of
//     trapping, as they did with the compilers the reference was written for.
#pragma once
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#define private public
#define protected public
#include "GRE.hpp"
#undef private
#undef protected

typedef GRE::Graph::DistributedGraph<GRE::Graph::GraphInCSR> RefGraph_t;

template <Dir dir>
inline void load_graph(RefGraph_t& g, GRE::COMM::Underlying& comm, GRE::Util::BufferPool& pool,
                       const std::string& prefix) {
  GRE::Graph::IngressParameters params(prefix, "ascii", "edgelists");
  GRE::Graph::GraphIngress<RefGraph_t>* ingress = new GRE::Graph::GraphIngress<RefGraph_t>(g, comm, pool);
  ingress->template ingress<dir>(params);
  g.isReady = true;
  ingress->finalize();
  g.lStat_nEdges = g.graph.get_num_edges();
  g.subGraphID = comm.rank();
  delete ingress;
}

inline std::vector<vid_t> load_roots(const std::string& prefix) {
  std::vector<vid_t> src;
  GRE::Util::loadFromFile(prefix + ".roots", src, 0);
  // loadFromFile keeps the leading count at src[0] (the drivers use src[1], usr/test_bfs.cpp:58)
  std::vector<vid_t> roots;
  if (src.empty()) return roots;
  const size_t cnt = (size_t)src[0];
  for (size_t i = 1; i <= cnt && i < src.size(); ++i) roots.push_back(src[i]);
  return roots;
}

inline bool write_array(const std::string& path, const void* data, size_t bytes) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  const size_t w = fwrite(data, 1, bytes, f);
  fclose(f);
  return w == bytes;
}

inline bool append_array(const std::string& path, const void* data, size_t bytes) {
  FILE* f = fopen(path.c_str(), "ab");
  if (!f) return false;
  const size_t w = fwrite(data, 1, bytes, f);
  fclose(f);
  return w == bytes;
}

// "GRE_RUN <name> <seconds> <supersteps>" lines are parsed by the Python side.
inline void report_run(const char* name, double seconds, long supersteps) {
  printf("GRE_RUN %s %.9f %ld\n", name, seconds, supersteps);
  fflush(stdout);
}
