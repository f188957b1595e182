// Counter-based, seeded RMAT edge generator shared by host (C++) and device (CUDA) code.
//
// The reference ships no graph data (data/edgelist.* are empty, data/graph.meta:1) and reads
// text edge lists `<prefix>.edges.<i>` + `<prefix>.meta` (Graph/GraphIngress.hpp:323-328,
// 570-591).  Every input of this project is therefore generated: edge e's quadrant at each
// recursion level comes from a hash of (seed, e, level), so the host and the GPU produce the
// same multiset of edges independently of thread count or launch shape.
//
// Quadrant probabilities a/b/c/d = 0.57/0.19/0.19/0.05 (Graph500 RMAT), 2^scale vertices,
// edgefactor * 2^scale raw edges; a seeded bijection on [0, 2^scale) then scatters hub ids.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GRE_HD __host__ __device__ __forceinline__
#else
#define GRE_HD inline
#endif

namespace gre {
namespace rmat {

// SplitMix64 finaliser (Steele, Lea, Flood 2014; public-domain reference by S. Vigna).
GRE_HD uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Params {
  uint32_t scale;
  uint64_t seed;
  uint32_t thr_a, thr_ab, thr_abc;  // cumulative quadrant thresholds on a 32-bit uniform
  uint64_t mask;
  uint64_t mul[3];
  uint64_t add[3];
  uint32_t shift;
};

inline Params make_params(uint32_t scale, uint64_t seed, double a = 0.57, double b = 0.19,
                          double c = 0.19) {
  Params p;
  p.scale = scale;
  p.seed = seed;
  const double two32 = 4294967296.0;
  p.thr_a = (uint32_t)(a * two32);
  p.thr_ab = (uint32_t)((a + b) * two32);
  p.thr_abc = (uint32_t)((a + b + c) * two32);
  p.mask = (scale >= 64) ? ~0ull : ((1ull << scale) - 1ull);
  for (int k = 0; k < 3; ++k) {
    p.mul[k] = splitmix64(seed ^ (0xA5A5ull + (uint64_t)k)) | 1ull;  // odd => bijective mod 2^s
    p.add[k] = splitmix64(seed ^ (0x5A5Aull + (uint64_t)k));
  }
  p.shift = scale / 2 + 1;
  return p;
}

// Seeded bijection on [0, 2^scale): three rounds of (odd multiply, xorshift, add), all mod 2^s.
GRE_HD uint64_t permute(const Params& p, uint64_t x) {
  for (int k = 0; k < 3; ++k) {
    x = (x * p.mul[k]) & p.mask;
    x ^= x >> p.shift;
    x = (x + p.add[k]) & p.mask;
  }
  return x;
}

// Raw RMAT edge e (before permutation): one 64-bit hash feeds two recursion levels.
GRE_HD void raw_edge(const Params& p, uint64_t e, uint64_t* u, uint64_t* v) {
  uint64_t su = 0, sv = 0;
  const uint64_t base = splitmix64(p.seed ^ splitmix64(e));
  for (uint32_t l = 0; l < p.scale; l += 2) {
    const uint64_t h = splitmix64(base + l);
    for (uint32_t t = 0; t < 2 && l + t < p.scale; ++t) {
      const uint32_t r = (uint32_t)(h >> (32 * t));
      uint32_t ub, vb;
      if (r < p.thr_a) { ub = 0; vb = 0; }
      else if (r < p.thr_ab) { ub = 0; vb = 1; }
      else if (r < p.thr_abc) { ub = 1; vb = 0; }
      else { ub = 1; vb = 1; }
      su = (su << 1) | ub;
      sv = (sv << 1) | vb;
    }
  }
  *u = su;
  *v = sv;
}

GRE_HD void edge(const Params& p, uint64_t e, uint32_t* u, uint32_t* v) {
  uint64_t ru, rv;
  raw_edge(p, e, &ru, &rv);
  *u = (uint32_t)permute(p, ru);
  *v = (uint32_t)permute(p, rv);
}

// SSSP weight of the undirected edge {u, v}: uniform in [1, 255], symmetric in (u, v) and
// independent of arc storage order.
GRE_HD uint32_t weight(uint64_t wseed, uint32_t u, uint32_t v) {
  const uint64_t lo = u < v ? u : v;
  const uint64_t hi = u < v ? v : u;
  return 1u + (uint32_t)(splitmix64(wseed ^ ((lo << 32) | hi)) % 255ull);
}

}  // namespace rmat
}  // namespace gre
