// ORACLE — test infrastructure only.  Force-included (-include) ahead of the reference headers
// when the reference GRE engine is compiled as a CPU oracle.
//
// g++ 13 rejects one line of the reference: DistributedGraph::get_lvid is a const member that
// calls the non-const HashIndex::value (Graph/DistributedGraph.hpp:48-53).  The call is
// non-dependent, so it is checked when the class template is parsed.  Declaring an explicit
// specialisation of HashIndex<vid_t, lvid_t> here, before the reference's DistributedGraph is
// seen, gives that call a const overload.  The specialisation is written for this project (a
// sorted vector with binary search) and has the interface the reference uses
// (Util/HashIndex.hpp:15-102); at one rank there are no agents, so it is never filled.
#pragma once
#include <stdint.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "Types.hpp"
#include "Util/HashIndex.hpp"

namespace GRE {
namespace Util {
template <>
class HashIndex<vid_t, lvid_t, int> {
 public:
  typedef std::pair<vid_t, lvid_t> entry_t;
  HashIndex(const vid_t invalid) : illegal_(invalid), entries_() {}
  lvid_t value(const vid_t key) const {
    std::vector<entry_t>::const_iterator it =
        std::lower_bound(entries_.begin(), entries_.end(), entry_t(key, 0));
    if (it != entries_.end() && it->first == key) return it->second;
    return (lvid_t)illegal_;
  }
  void buildFromArray(std::vector<vid_t>& keys) { buildFromArray(keys, 0, (long)keys.size()); }
  void buildFromArray(std::vector<vid_t>& keys, const long begin) {
    buildFromArray(keys, begin, (long)keys.size() - begin);
  }
  void buildFromArray(std::vector<vid_t>& keys, const long begin, const long count) {
    entries_.clear();
    for (long i = 0; i < count; i++) entries_.push_back(entry_t(keys[begin + i], (lvid_t)(begin + i)));
    std::sort(entries_.begin(), entries_.end());
  }
  void clear() { entries_.clear(); }
  void reset() { clear(); }
  void load() {}
  void save() {}

 private:
  vid_t illegal_;
  std::vector<entry_t> entries_;
};
}  // namespace Util
}  // namespace GRE
