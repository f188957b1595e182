// Host-side graph construction: seeded RMAT generation, GRE text edge-list files, and the
// `.meta` + `.edges.<i>` loader that feeds the device CSR/CSC.
//
// File format (restated from the reference loader, Graph/GraphIngress.hpp):
//   <prefix>.meta       "nV nE"                                  (GraphIngress.hpp:323-328)
//   <prefix>.edges.<i>  one "src dst" per line, base-10; lines that are empty or start with
//                       '#' are skipped                            (GraphIngress.hpp:581-588)
//   files are read for i = 0, 1, 2, ... until one fails to open   (GraphIngress.hpp:570-578)
//   <prefix>.roots      "count v1 v2 ..."                          (Util/Util.hpp:140-157)
// Arc order of the CSR the reference builds: source-major, and within a source the order the
// arcs were read (Graph/LocalGraph.hpp:66-107).  The loader here keeps exactly that order.
//
// Where the reference silently accepts bad input (ids >= nV write out of bounds, text after
// the numbers is ignored), this loader returns GRE_INVALID_ARG / GRE_IO_ERROR instead.
#include <errno.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <parallel/algorithm>
#include <string>
#include <vector>

#include "../../include/gre_gpu.h"
#include "host_api.hpp"
#include "rmat.hpp"

namespace gre {

// ---------------------------------------------------------------------------------------------
// RMAT generation on the host (OpenMP).  Same edges as the device generator (rmat.hpp).
// ---------------------------------------------------------------------------------------------
int host_rmat_csr(uint32_t scale, uint32_t edgefactor, uint64_t seed, int symmetric, HostCSR* out) {
  if (scale == 0 || scale > 31 || edgefactor == 0) return GRE_INVALID_ARG;
  const rmat::Params p = rmat::make_params(scale, seed);
  const uint64_t n = 1ull << scale;
  const uint64_t m_raw = (uint64_t)edgefactor << scale;
  const uint64_t nkeys = symmetric ? 2 * m_raw : m_raw;
  std::vector<uint64_t> keys;
  try {
    keys.resize(nkeys);
  } catch (...) {
    return GRE_OOM;
  }
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)m_raw; ++e) {
    uint32_t u, v;
    rmat::edge(p, (uint64_t)e, &u, &v);
    // self loops are marked with an all-ones key and dropped after the sort
    const uint64_t self = (u == v) ? ~0ull : 0ull;
    keys[e] = (((uint64_t)u << 32) | v) | self;
    if (symmetric) keys[m_raw + e] = (((uint64_t)v << 32) | u) | self;
  }
  __gnu_parallel::sort(keys.begin(), keys.end());
  auto last = std::unique(keys.begin(), keys.end());
  while (last != keys.begin() && *(last - 1) == ~0ull) --last;
  const uint64_t m = (uint64_t)(last - keys.begin());
  out->n = n;
  out->m = m;
  out->off.assign(n + 1, 0);
  out->col.resize(m);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)m; ++i) out->col[i] = (uint32_t)(keys[i] & 0xffffffffull);
  // row offsets: first arc index of each source (keys are sorted by source)
  for (uint64_t i = 0; i < m; ++i) out->off[(keys[i] >> 32) + 1]++;
  for (uint64_t v = 0; v < n; ++v) out->off[v + 1] += out->off[v];
  return GRE_SUCCESS;
}

// ---------------------------------------------------------------------------------------------
// Text writer: <prefix>.meta and <prefix>.edges.<i>, source u goes to file (u % nfiles).
// Splitting by source keeps multi-rank reference runs correct (outdegrees are counted by the
// reading rank, GraphIngress.hpp:591).
// ---------------------------------------------------------------------------------------------
static char* put_u64(char* p, uint64_t x) {
  char tmp[24];
  int k = 0;
  do {
    tmp[k++] = (char)('0' + x % 10);
    x /= 10;
  } while (x);
  while (k) *p++ = tmp[--k];
  return p;
}

int host_write_edgelists(const char* prefix, uint64_t n, uint64_t m, const uint64_t* off,
                         const uint32_t* col, uint32_t nfiles) {
  if (!prefix || nfiles == 0) return GRE_INVALID_ARG;
  {
    std::string meta = std::string(prefix) + ".meta";
    FILE* f = fopen(meta.c_str(), "w");
    if (!f) return GRE_IO_ERROR;
    fprintf(f, "%llu %llu\n", (unsigned long long)n, (unsigned long long)m);
    if (fclose(f) != 0) return GRE_IO_ERROR;
  }
  int status = GRE_SUCCESS;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t fi = 0; fi < (int64_t)nfiles; ++fi) {
    std::string name = std::string(prefix) + ".edges." + std::to_string(fi);
    FILE* f = fopen(name.c_str(), "w");
    if (!f) {
#pragma omp atomic write
      status = GRE_IO_ERROR;
      continue;
    }
    const size_t cap = 1 << 22;
    std::vector<char> buf(cap + 64);
    char* p = buf.data();
    for (uint64_t u = (uint64_t)fi; u < n; u += nfiles) {
      for (uint64_t a = off[u]; a < off[u + 1]; ++a) {
        p = put_u64(p, u);
        *p++ = ' ';
        p = put_u64(p, col[a]);
        *p++ = '\n';
        if ((size_t)(p - buf.data()) >= cap) {
          fwrite(buf.data(), 1, p - buf.data(), f);
          p = buf.data();
        }
      }
    }
    fwrite(buf.data(), 1, p - buf.data(), f);
    if (fclose(f) != 0) {
#pragma omp atomic write
      status = GRE_IO_ERROR;
    }
  }
  return status;
}

int host_write_roots(const char* prefix, const uint32_t* roots, uint32_t count) {
  std::string name = std::string(prefix) + ".roots";
  FILE* f = fopen(name.c_str(), "w");
  if (!f) return GRE_IO_ERROR;
  fprintf(f, "%u\n", count);
  for (uint32_t i = 0; i < count; ++i) fprintf(f, "%u\n", roots[i]);
  return fclose(f) == 0 ? GRE_SUCCESS : GRE_IO_ERROR;
}

int host_read_roots(const char* prefix, std::vector<uint32_t>* roots) {
  std::string name = std::string(prefix) + ".roots";
  FILE* f = fopen(name.c_str(), "r");
  if (!f) return GRE_IO_ERROR;
  unsigned long long cnt = 0;
  if (fscanf(f, "%llu", &cnt) != 1) {
    fclose(f);
    return GRE_IO_ERROR;
  }
  roots->clear();
  for (unsigned long long i = 0; i < cnt; ++i) {
    unsigned long long v;
    if (fscanf(f, "%llu", &v) != 1) {
      fclose(f);
      return GRE_IO_ERROR;
    }
    roots->push_back((uint32_t)v);
  }
  fclose(f);
  return GRE_SUCCESS;
}

// Stable counting sort of (src, dst) by src: source-major CSR, input order within a source
// (GraphInCSR::build, LocalGraph.hpp:66-107).  When `by_dst` is set the roles swap and the
// result is the reverse CSR (GraphInCSR::rbuild, LocalGraph.hpp:112-156).
void host_build_csr(uint64_t n, const std::vector<uint32_t>& src, const std::vector<uint32_t>& dst,
                    bool by_dst, std::vector<uint64_t>* off, std::vector<uint32_t>* col) {
  const std::vector<uint32_t>& key = by_dst ? dst : src;
  const std::vector<uint32_t>& val = by_dst ? src : dst;
  const uint64_t m = key.size();
  off->assign(n + 1, 0);
  for (uint64_t i = 0; i < m; ++i) (*off)[key[i] + 1]++;
  for (uint64_t v = 0; v < n; ++v) (*off)[v + 1] += (*off)[v];
  col->resize(m);
  std::vector<uint64_t> cur(off->begin(), off->end() - 1);
  for (uint64_t i = 0; i < m; ++i) (*col)[cur[key[i]]++] = val[i];
}

}  // namespace gre

// ---------------------------------------------------------------------------------------------
// C ABI (host-only utilities)
// ---------------------------------------------------------------------------------------------
extern "C" {

int gre_rmat_host(uint32_t scale, uint32_t edgefactor, uint64_t seed, int symmetric,
                  uint64_t* n, uint64_t* m, uint64_t** row_off, uint32_t** col) {
  if (!n || !m || !row_off || !col) return GRE_NULL;
  gre::HostCSR csr;
  int st = gre::host_rmat_csr(scale, edgefactor, seed, symmetric, &csr);
  if (st) return st;
  *n = csr.n;
  *m = csr.m;
  *row_off = (uint64_t*)malloc(sizeof(uint64_t) * (csr.n + 1));
  *col = (uint32_t*)malloc(sizeof(uint32_t) * (csr.m ? csr.m : 1));
  if (!*row_off || !*col) {
    free(*row_off);
    free(*col);
    *row_off = nullptr;
    *col = nullptr;
    return GRE_OOM;
  }
  memcpy(*row_off, csr.off.data(), sizeof(uint64_t) * (csr.n + 1));
  if (csr.m) memcpy(*col, csr.col.data(), sizeof(uint32_t) * csr.m);
  return GRE_SUCCESS;
}

void gre_host_free(void* p) { free(p); }

int gre_write_edgelists(const char* prefix, uint64_t n, uint64_t m, const uint64_t* row_off,
                        const uint32_t* col, uint32_t nfiles) {
  if (!prefix || !row_off || (m && !col)) return GRE_NULL;
  if (row_off[n] != m) return GRE_INVALID_ARG;
  return gre::host_write_edgelists(prefix, n, m, row_off, col, nfiles);
}

int gre_write_roots(const char* prefix, const uint32_t* roots, uint32_t count) {
  if (!prefix || (count && !roots)) return GRE_NULL;
  return gre::host_write_roots(prefix, roots, count);
}

int gre_read_roots(const char* prefix, uint32_t* roots, uint32_t capacity, uint32_t* count) {
  if (!prefix || !count) return GRE_NULL;
  std::vector<uint32_t> r;
  int st = gre::host_read_roots(prefix, &r);
  if (st) return st;
  *count = (uint32_t)r.size();
  if (roots)
    for (uint32_t i = 0; i < r.size() && i < capacity; ++i) roots[i] = r[i];
  return r.size() > capacity && roots ? GRE_NOBUFFER : GRE_SUCCESS;
}

uint32_t gre_sssp_weight(uint64_t wseed, uint32_t u, uint32_t v) {
  return gre::rmat::weight(wseed, u, v);
}

}  // extern "C"
