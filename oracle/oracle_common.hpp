// ORACLE — test infrastructure only.  Nothing in the product (graphine_b200/, include/) may
// include, link or call this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg use it, as a checker.
//
// Input definitions shared by the oracle's restatement and the reference harness drivers.
// Restated independently of the product's generator so that a mismatch shows up as a parity
// failure instead of being hidden by shared code.
#pragma once
#include <stdint.h>

namespace gre_oracle {

// SplitMix64 finaliser (public-domain reference by S. Vigna).
static inline uint64_t mix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// SSSP weight of the undirected edge {u, v}: 1 + H(seed, min, max) % 255, i.e. uniform in
// [1, 255].  Replaces the reference's unseeded rand()%65535 per CSR slot
// (Graph/DistributedGraph.hpp:219-226), which cannot be reproduced across runs.
static inline uint32_t sssp_weight(uint64_t wseed, uint64_t u, uint64_t v) {
  const uint64_t lo = u < v ? u : v;
  const uint64_t hi = u < v ? v : u;
  return 1u + (uint32_t)(mix64(wseed ^ ((lo << 32) | hi)) % 255ull);
}

}  // namespace gre_oracle
