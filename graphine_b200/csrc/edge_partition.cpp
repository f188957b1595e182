// Offline edge partitioner (host only, no GPU): the reference's single-process EdgePartition
// (include/Graph/GraphIngress.hpp:1272-1452, driven by usr/debug/test_graphPar.cpp), which splits
// a graph's edge lists into P edge sets for an np = P run and writes them in the layout that run
// loads (GraphIngress.hpp:1024-1071) and that gre_graph_load_parts reads here.
//
// Decision per edge (u, v), in the order the reference streams them (pass p = 0..P-1 reads
// <prefix>.edges.p, .edges.(p+P), ... until a file is missing; lines empty or starting with '#'
// are skipped; "u v" parsed as two base-10 integers): greedy vertex-cut placement with a balance
// term (GraphIngress.hpp:1426-1449).  For every part i, with lo / hi the smallest / largest edge
// count so far,
//     score_i = (hi - count_i) / (1 + (hi - lo)) + [u already a source in i] + [v already a head in i]
// and among the parts within 1e-4 of the best score the one at position (u + v) mod (their number)
// in increasing part order takes the edge.  The scores are computed with the reference's
// operations in its order, so ties resolve the same way and the parts are the same edges in the
// same order.
//
// Files (P = nparts):
//   <prefix>.part.P.r        edges of part r as binary (uint64 u, uint64 v) pairs, in decision
//                            order (written only for parts that received an edge)
//   <prefix>.outdegree.P.p   int32 per master of pass p (nv / P + (nv % P > p) of them): the
//                            edges read in pass p counted at u / P, where that index is in range
//   <prefix>.scatterMap.P.p  for every part j != p in order: int64 bit count, then count / 8 + 8
//                            bytes of the bitmap of the indices u / P of pass p's edges placed in j
//                            (the bit count is that of pass 0, the largest, for every pass)
// Differences from the reference, where its behaviour is undefined or depends on history: files
// are written afresh (the reference appends to existing ones); the scatter-map bytes past the
// bitmap's 64-bit words (written from beyond the reference's allocation when count % 64 >= 8) are
// zeros; an edge whose vertex id is not below the .meta vertex count is an error, as is P outside
// 1..64 (the reference's per-vertex part sets are 64 bits wide, Config/UsrConfig.hpp:17).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gre_gpu.h"
#include "host_api.hpp"

namespace gre {
namespace {

class GreedyEdgeSplit {
 public:
  GreedyEdgeSplit(uint32_t nparts, uint64_t nv) : P_(nparts), as_src_(nv, 0), as_dst_(nv, 0), count_(nparts, 0), score_(nparts) {}

  uint32_t place(uint64_t u, uint64_t v) {
    uint64_t lo = count_[0], hi = count_[0];
    for (uint32_t i = 1; i < P_; ++i) {
      lo = count_[i] < lo ? count_[i] : lo;
      hi = count_[i] > hi ? count_[i] : hi;
    }
    const double base = 1.0 + (double)(hi - lo);
    double best = 0.0;
    for (uint32_t i = 0; i < P_; ++i) {
      const double balance = (double)(hi - count_[i]) / base;
      score_[i] = balance + (((as_src_[u] >> i) & 1ull) ? 1.0 : 0.0) + (((as_dst_[v] >> i) & 1ull) ? 1.0 : 0.0);
      if (i == 0 || score_[i] > best) best = score_[i];
    }
    uint32_t ties[64];
    uint32_t nties = 0;
    for (uint32_t i = 0; i < P_; ++i)
      if (std::fabs(best - score_[i]) < 1e-4) ties[nties++] = i;
    const uint32_t r = ties[(u + v) % nties];
    ++count_[r];
    as_src_[u] |= 1ull << r;
    as_dst_[v] |= 1ull << r;
    return r;
  }

  const std::vector<uint64_t>& counts() const { return count_; }

 private:
  uint32_t P_;
  std::vector<uint64_t> as_src_, as_dst_;  // bit i: the vertex is a source / a head of an edge of part i
  std::vector<uint64_t> count_;
  std::vector<double> score_;
};

// Edges of one part, written in blocks as the reference flushes them (2^23 edges).
class PartWriter {
 public:
  explicit PartWriter(std::string name) : name_(std::move(name)) {}
  int add(uint64_t u, uint64_t v) {
    buf_.push_back(u);
    buf_.push_back(v);
    return buf_.size() >= 2 * kBlock ? flush() : GRE_SUCCESS;
  }
  int flush() {
    if (buf_.empty()) return GRE_SUCCESS;
    if (!out_) {
      out_.reset(new std::ofstream(name_.c_str(), std::ios::out | std::ios::binary | std::ios::trunc));
      if (!*out_) {
        set_error("gre_partition_edges: cannot write %s", name_.c_str());
        return GRE_IO_ERROR;
      }
    }
    out_->write(reinterpret_cast<const char*>(buf_.data()), (std::streamsize)(sizeof(uint64_t) * buf_.size()));
    buf_.clear();
    if (!*out_) {
      set_error("gre_partition_edges: write to %s failed", name_.c_str());
      return GRE_IO_ERROR;
    }
    return GRE_SUCCESS;
  }

 private:
  static const size_t kBlock = 1u << 23;
  std::string name_;
  std::vector<uint64_t> buf_;
  std::unique_ptr<std::ofstream> out_;
};

// One file from a list of (data, bytes) pieces.
int write_file(const std::string& name, const std::vector<std::pair<const void*, size_t>>& pieces) {
  std::ofstream f(name.c_str(), std::ios::out | std::ios::binary | std::ios::trunc);
  if (!f) {
    set_error("gre_partition_edges: cannot write %s", name.c_str());
    return GRE_IO_ERROR;
  }
  for (const auto& pc : pieces)
    if (pc.second) f.write(reinterpret_cast<const char*>(pc.first), (std::streamsize)pc.second);
  if (!f) {
    set_error("gre_partition_edges: write to %s failed", name.c_str());
    return GRE_IO_ERROR;
  }
  return GRE_SUCCESS;
}

}  // namespace
}  // namespace gre

extern "C" int gre_partition_edges(const char* prefix, uint32_t nparts, uint64_t* part_edges) {
  using namespace gre;
  if (!prefix) return GRE_NULL;
  clear_error();
  if (nparts < 1 || nparts > 64) {
    set_error("gre_partition_edges: %u parts (1..64)", nparts);
    return GRE_INVALID_ARG;
  }
  const std::string pre(prefix);
  uint64_t nv = 0, ne = 0;
  {
    std::ifstream meta((pre + ".meta").c_str());
    if (!(meta >> nv >> ne)) {
      set_error("gre_partition_edges: cannot read %s.meta", prefix);
      return GRE_IO_ERROR;
    }
  }
  const uint64_t P = nparts;
  GreedyEdgeSplit split(nparts, nv);
  std::vector<std::unique_ptr<PartWriter>> parts;
  for (uint64_t r = 0; r < P; ++r)
    parts.emplace_back(new PartWriter(pre + ".part." + std::to_string(P) + "." + std::to_string(r)));
  // bitmaps of the scatter maps: pass 0's master count of bits, plus a zero word for the bytes
  // written past the last full word
  const uint64_t bits = nv / P + (nv % P > 0 ? 1 : 0);
  const uint64_t words = bits / 64 + 2;
  const size_t map_bytes = (size_t)(bits / 8 + 8);
  const int64_t bits_field = (int64_t)bits;
  for (uint64_t p = 0; p < P; ++p) {
    const uint64_t masters = nv / P + (nv % P > p ? 1 : 0);
    std::vector<int32_t> outdeg(masters, 0);
    std::vector<std::vector<uint64_t>> scatter(P, std::vector<uint64_t>(words, 0));
    for (uint64_t i = p;; i += P) {
      std::ifstream f((pre + ".edges." + std::to_string(i)).c_str());
      if (!f) break;
      std::string line;
      while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        char* end = nullptr;
        const uint64_t u = strtoull(line.c_str(), &end, 10);
        const uint64_t v = strtoull(end, nullptr, 10);
        if (u >= nv || v >= nv) {
          set_error("gre_partition_edges: edge (%llu, %llu) in %s.edges.%llu: vertex ids must be below %llu",
                    (unsigned long long)u, (unsigned long long)v, prefix, (unsigned long long)i, (unsigned long long)nv);
          return GRE_INVALID_ARG;
        }
        const uint32_t r = split.place(u, v);
        int st = parts[r]->add(u, v);
        if (st) return st;
        const uint64_t ls = u / P;  // u's index among its rank's masters
        if (ls < masters) ++outdeg[ls];
        scatter[r][ls >> 6] |= 1ull << (ls & 63u);
      }
    }
    int st = write_file(pre + ".outdegree." + std::to_string(P) + "." + std::to_string(p),
                        {{outdeg.data(), sizeof(int32_t) * outdeg.size()}});
    if (st) return st;
    std::vector<std::pair<const void*, size_t>> pieces;
    for (uint64_t j = 0; j < P; ++j) {
      if (j == p) continue;
      pieces.push_back({&bits_field, sizeof bits_field});
      pieces.push_back({scatter[j].data(), map_bytes});
    }
    st = write_file(pre + ".scatterMap." + std::to_string(P) + "." + std::to_string(p), pieces);
    if (st) return st;
  }
  for (auto& w : parts) {
    int st = w->flush();
    if (st) return st;
  }
  if (part_edges)
    for (uint64_t r = 0; r < P; ++r) part_edges[r] = split.counts()[r];
  return GRE_SUCCESS;
}

