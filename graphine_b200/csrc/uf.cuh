// Lock-free union-find with min-key hooking (Jayanti and Tarjan style concurrent union-find, as
// in ECL-CC, Jaiganesh and Burtscher 2018): used by the one-GPU CC (cc.cu) and by the local
// phase of the partitioned CC (partition.cu).  A root is only ever linked under a root of
// smaller key (atomicCAS on the larger root's parent), so every tree's root holds the smallest
// key of its members.
#pragma once
#include <vector>

#include "gre_internal.cuh"

namespace gre {

__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x) {
  uint32_t p = parent[x];
  while (p != x) {
    const uint32_t gp = parent[p];
    if (gp != p) parent[x] = gp;  // path halving (benign race: gp is an ancestor)
    x = p;
    p = gp;
  }
  return x;
}

// key(x): the caller's id of vertex x (null map: x itself) - roots are linked by it
__device__ __forceinline__ uint32_t uf_key(const uint32_t* __restrict__ key, uint32_t x) { return key ? __ldg(key + x) : x; }

__device__ __forceinline__ void uf_union(uint32_t* parent, const uint32_t* __restrict__ key, uint32_t a, uint32_t b) {
  while (true) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return;
    const bool a_hi = uf_key(key, a) > uf_key(key, b);
    const uint32_t hi = a_hi ? a : b;
    const uint32_t lo = a_hi ? b : a;
    if (atomicCAS(parent + hi, hi, lo) == hi) return;
    // hi gained a parent meanwhile: retry from the new roots
    a = hi;
    b = lo;
  }
}

// kernels defined in cc.cu
__global__ void k_uf_init(uint64_t n, uint32_t* __restrict__ parent);
__global__ void k_uf_compress(uint64_t n, uint32_t* parent, uint64_t stride, uint32_t* __restrict__ sample, uint32_t nsample);
__global__ void k_uf_skipbits(uint64_t n, const uint32_t* __restrict__ parent, const uint64_t* __restrict__ off, uint32_t c,
                              uint32_t k, uint32_t* __restrict__ skip, unsigned long long* __restrict__ counts);

// The most frequent root among `ns` sampled roots (Afforest's guess of the largest component).
uint32_t uf_most_frequent(std::vector<uint32_t>& roots, uint32_t ns);

}  // namespace gre
