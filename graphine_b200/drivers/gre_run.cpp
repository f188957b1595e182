// gre_run — drop-in for the reference example drivers (usr/test_pagerank.cpp, test_bfs.cpp,
// test_sssp.cpp, test_cc.cpp, test_cIn.cpp, test_bc.cpp) on libgre_gpu.so, written against
// gre/gre.hpp.
//
//   gre_run <pagerank|pagerank_iter|pagerank_delta|bfs|sssp|sssp1|cc|cin|bc> <prefix> [ascii] [edgelists]
//
// Same inputs (<prefix>.meta, <prefix>.edges.<i>, <prefix>.roots, source = the first root as
// the reference's src[1]) and the same per-superstep lines the reference engine prints
// ("Superstep-k: Number of active vertices...N", Engine.hpp:396-398), then the iteration
// count and the run time.  Differences: one GPU, no MPI; SSSP weights come from the seeded
// weight function (environment GRE_WSEED, default 1) instead of unseeded rand(); BC runs all
// roots of the file and accumulates them.  Exit status 0 on success, the gre status otherwise.
//
//   gre_run <part_bfs|part_sssp|part_cc|part_pagerank|part_pagerank_iter> <prefix> --ranks P --rank r --id-file F [--device d]
//
// One rank of an np = P job over P GPUs (the reference's mpirun -np P): every rank loads the
// graph, keeps its part (gre/gre.hpp PartitionedGraph) and runs over the library's NCCL
// communicator.  Rank 0 writes the communicator id to F, the others wait for it (up to 120 s).
// Every rank prints the same lines; rank 0's are the job's.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gre/gre.hpp"

static void print_supersteps(const gre_stats& st) {
  for (uint32_t i = 0; i < st.n_recorded; ++i)
    printf("Superstep-%u: Number of active vertices...%llu\n", i, (unsigned long long)st.active[i]);
}

// The communicator id through a file: rank 0 writes it whole (temporary name, then rename).
static std::vector<uint8_t> shared_id(const std::string& path, int rank) {
  if (rank == 0) {
    std::vector<uint8_t> id = gre::Underlying::uniqueId();
    const std::string tmp = path + ".tmp";
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f || fwrite(id.data(), 1, id.size(), f) != id.size() || fclose(f) != 0 || rename(tmp.c_str(), path.c_str()))
      throw gre::Error(GRE_IO_ERROR, "cannot write the id file " + path);
    return id;
  }
  for (int i = 0; i < 12000; ++i) {  // 120 s
    if (FILE* f = fopen(path.c_str(), "rb")) {
      std::vector<uint8_t> id(128);
      const size_t got = fread(id.data(), 1, id.size(), f);
      fclose(f);
      if (got == id.size()) return id;
    }
    std::this_thread::sleep_for(std::chrono::milliseconds(10));
  }
  throw gre::Error(GRE_TIMEOUT, "no id file " + path + " from rank 0");
}

static int run_partitioned(const std::string& algo, const std::string& prefix, int argc, char** argv) {
  if (algo != "part_bfs" && algo != "part_sssp" && algo != "part_cc" && algo != "part_pagerank" &&
      algo != "part_pagerank_iter") {
    fprintf(stderr, "unknown algorithm %s\n", algo.c_str());
    return 2;
  }
  int ranks = 1, rank = 0, device = 0;
  std::string id_file;
  for (int i = 3; i + 1 < argc; i += 2) {
    const std::string k(argv[i]);
    if (k == "--ranks") ranks = atoi(argv[i + 1]);
    else if (k == "--rank") rank = atoi(argv[i + 1]);
    else if (k == "--device") device = atoi(argv[i + 1]);
    else if (k == "--id-file") id_file = argv[i + 1];
    else {
      fprintf(stderr, "unknown option %s\n", k.c_str());
      return 2;
    }
  }
  if (ranks < 1 || rank < 0 || rank >= ranks || id_file.empty()) {
    fprintf(stderr, "need --ranks P --rank r (0 <= r < P) --id-file F\n");
    return 2;
  }
  gre::Underlying comm(shared_id(id_file, rank), ranks, rank, device);
  gre_stats st{};
  {
    gre::DistributedGraph g;
    if (algo == "part_bfs" || algo == "part_cc") g.ingress<gre::InOut>(prefix, "ascii", "edgelists", false, true, device);
    else g.ingress<gre::Out>(prefix, "ascii", "edgelists", false, true, device);
    if (algo == "part_sssp") {
      const char* ws = getenv("GRE_WSEED");
      g.loadEdgePropertyHash(ws ? strtoull(ws, nullptr, 10) : 1);
    }
    gre::PartitionedGraph part(g, comm);
    uint32_t root = 0;
    if (algo == "part_bfs" || algo == "part_sssp") {
      std::vector<uint32_t> roots(1024);
      uint32_t nroots = 0;
      int s = gre_read_roots(prefix.c_str(), roots.data(), (uint32_t)roots.size(), &nroots);
      if ((s != GRE_SUCCESS && s != GRE_NOBUFFER) || nroots == 0) {
        fprintf(stderr, "Err in reading src vertex from file.\n");
        return s ? s : GRE_IO_ERROR;
      }
      root = roots[0];
    }
    if (algo == "part_bfs") {
      std::vector<int32_t> level = part.bfs(root, &st);
      print_supersteps(st);
      long reached = 0;
      for (int32_t l : level) reached += l >= 0;
      printf("Reached vertices: %ld\n", reached);
    } else if (algo == "part_sssp") {
      std::vector<uint32_t> dist = part.sssp(root, &st);
      long reached = 0;
      unsigned long long total = 0;
      for (uint32_t d : dist)
        if (d != 0xffffffffu) {
          ++reached;
          total += d;
        }
      printf("Reached vertices: %ld\nSum of distances: %llu\n", reached, total);
    } else if (algo == "part_cc") {
      std::vector<uint32_t> label = part.cc(&st);
      long comps = 0;
      for (size_t v = 0; v < label.size(); ++v) comps += label[v] == v;
      printf("Number of components: %ld\n", comps);
    } else {
      std::vector<double> pr = part.pagerank(algo == "part_pagerank_iter", 0.85, algo == "part_pagerank" ? 10 : 20, &st);
      double sum = 0;
      for (double x : pr) sum += x;
      printf("Sum of pr: %.15g\n", sum);
    }
  }
  printf("B200 | rank %d of %d | Iteration count: %u\n", rank, ranks, st.supersteps);
  printf("B200 | Use time: %gs\n", st.device_ms * 1e-3);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s pagerank|pagerank_iter|pagerank_delta|bfs|sssp|sssp1|cc|cin|bc prefix [ascii] "
                    "[edgelists|partition [nparts]]\n"
                    "       %s part_bfs|part_sssp|part_cc|part_pagerank|part_pagerank_iter prefix --ranks P --rank r --id-file F [--device d]\n"
                    "       %s graphpar prefix nparts\n",
            argv[0], argv[0], argv[0]);
    return 2;
  }
  const std::string algo(argv[1]), prefix(argv[2]);
  if (algo == "graphpar") {  // the offline partitioner, as usr/debug/test_graphPar.cpp
    const uint32_t nparts = argc > 3 ? (uint32_t)strtoul(argv[3], nullptr, 10) : 0u;
    std::vector<uint64_t> counts(nparts ? nparts : 1);
    const int st = gre_partition_edges(prefix.c_str(), nparts, counts.data());
    if (st) {
      fprintf(stderr, "%s\n", gre_last_error());
      return st;
    }
    for (uint32_t r = 0; r < nparts; ++r) printf("part %u: %llu edges\n", r, (unsigned long long)counts[r]);
    return 0;
  }
  if (algo.rfind("part_", 0) == 0) {
    try {
      return run_partitioned(algo, prefix, argc, argv);
    } catch (const gre::Error& e) {
      fprintf(stderr, "%s\n", e.what());
      return e.status;
    }
  }
  try {
    gre::DistributedGraph g;
    const bool in_out = algo == "bfs" || algo == "cc" || algo == "bc" || algo == "cin";
    // format and method as the reference drivers take them (usr/test_bfs.cpp:40-47); a saved
    // partition set also needs its part count (the reference's rank count)
    const std::string format = argc > 3 ? argv[3] : "ascii";
    const std::string method = argc > 4 ? argv[4] : "edgelists";
    const uint32_t nparts = argc > 5 ? (uint32_t)strtoul(argv[5], nullptr, 10) : 1u;
    if (in_out) g.ingress<gre::InOut>(prefix, format, method, false, false, 0, nparts);
    else g.ingress<gre::Out>(prefix, format, method, false, false, 0, nparts);
    std::vector<uint32_t> roots(1024);
    uint32_t nroots = 0;
    if (algo == "bfs" || algo == "sssp" || algo == "sssp1" || algo == "bc") {
      int s = gre_read_roots(prefix.c_str(), roots.data(), (uint32_t)roots.size(), &nroots);
      if ((s != GRE_SUCCESS && s != GRE_NOBUFFER) || nroots == 0) {
        fprintf(stderr, "Err in reading src vertex from file.\n");
        return s ? s : GRE_IO_ERROR;
      }
      roots.resize(nroots < roots.size() ? nroots : roots.size());
    }
    gre::SourceVertexSet src;
    gre_stats st{};
    if (algo == "pagerank" || algo == "pagerank_iter") {
      src.setALL();
      gre::PageRank pr(g, algo == "pagerank_iter");
      gre::SynchronousEngine<gre::PageRank> engine(g, pr);
      engine.initialize();
      engine.configMaxSupersteps(algo == "pagerank" ? 10 : 20);  // usr/test_pagerank.cpp:70
      engine.run<gre::Out>(src);
      st = engine.stats();
      print_supersteps(st);
      printf("Sum of pr: %.15g\n", st.plugin_value);  // the plugin's output_statistics
    } else if (algo == "pagerank_delta") {  // usr/test_pagerank.cpp:22 with the PageRank_delta typedef
      src.setALL();
      gre::PageRank_delta pr(g);
      gre::SynchronousEngine<gre::PageRank_delta> engine(g, pr);
      engine.run<gre::Out>(src);
      st = engine.stats();
      double sum = 0;
      for (double x : pr.pr) sum += x;
      print_supersteps(st);
      printf("Sum of pr: %.15g\n", sum);
    } else if (algo == "sssp1") {
      const char* ws = getenv("GRE_WSEED");
      g.loadEdgePropertyHash(ws ? strtoull(ws, nullptr, 10) : 1);
      src.addVertex(roots[0], g);
      gre::SSSP1 sssp(g);
      gre::SynchronousEngine<gre::SSSP1> engine(g, sssp);
      engine.configMaxSupersteps(128);
      engine.run<gre::Out>(src);
      st = engine.stats();
      print_supersteps(st);
    } else if (algo == "cin") {  // usr/test_cIn.cpp
      src.setALL();
      gre::CountIn cin(g);
      gre::SynchronousEngine<gre::CountIn> engine(g, cin);
      engine.configMaxSupersteps(1);
      engine.run<gre::In>(src);
      st = engine.stats();
      print_supersteps(st);
      printf("Number of in edges: %llu\n", (unsigned long long)st.plugin_count);  // output_statistics
    } else if (algo == "bfs") {
      src.addVertex(roots[0], g);
      gre::BFS bfs(g);
      gre::SynchronousEngine<gre::BFS> engine(g, bfs);
      engine.run<gre::In>(src);  // usr/test_bfs.cpp:69
      st = engine.stats();
      print_supersteps(st);
    } else if (algo == "sssp") {
      const char* ws = getenv("GRE_WSEED");
      g.loadEdgePropertyHash(ws ? strtoull(ws, nullptr, 10) : 1);
      src.addVertex(roots[0], g);
      gre::SSSP sssp(g);
      gre::SynchronousEngine<gre::SSSP> engine(g, sssp);
      engine.configMaxSupersteps(128);  // usr/test_sssp.cpp:64
      engine.run<gre::Out>(src);
      st = engine.stats();
      print_supersteps(st);
    } else if (algo == "cc") {
      src.setALL();
      gre::ConnectedComponents cc(g);
      gre::SynchronousEngine<gre::ConnectedComponents> engine(g, cc);
      engine.run<gre::InOut>(src);
      st = engine.stats();
      print_supersteps(st);
      printf("Number of components: %llu\n", (unsigned long long)st.plugin_count);  // output_statistics
    } else if (algo == "bc") {
      for (uint32_t r : roots) src.addVertex(r, g);
      gre::BC bc(g);
      gre::SynchronousEngine<gre::BC> engine(g, bc);
      engine.run<gre::Out>(src);
      st = engine.stats();
    } else {
      fprintf(stderr, "unknown algorithm %s\n", algo.c_str());
      return 2;
    }
    printf("B200 | Iteration count: %u\n", st.supersteps);
    printf("B200 | Use time: %gs\n", st.device_ms * 1e-3);
  } catch (const gre::Error& e) {
    fprintf(stderr, "%s\n", e.what());
    return e.status;
  }
  return 0;
}
