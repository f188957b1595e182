// ORACLE — test infrastructure only.  Host-only input generation for the checker and for the
// CPU reference arm of bench.py, so that neither loads the product library.
//
// What it restates (an independent rewrite of the input definitions, not a call into the
// product): the seeded RMAT generator the product's graphs come from (Graph500 quadrant
// probabilities a/b/c/d = 0.57/0.19/0.19/0.05; edge e's two quadrant bits per 64-bit hash of
// (seed, e, level pair); a seeded three-round bijection on [0, 2^scale) that scatters hub ids;
// self loops and duplicates dropped; symmetrised on request), the reference's text edge-list
// format (`<prefix>.meta` "nV nE", Graph/GraphIngress.hpp:323-328; `<prefix>.edges.<i>` one
// "u v" per line, files enumerated i = 0, 1, ... until one fails to open,
// GraphIngress.hpp:570-591; source u in file u % nfiles), the `.roots` list with its leading
// count (Util/Util.hpp:140-157), and the harness SSSP weight of every CSR arc.
//
// A CPU test checks that these graphs equal the product's host generator arc for arc.
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <parallel/algorithm>
#include <string>
#include <vector>

#include "oracle_common.hpp"

namespace {

using gre_oracle::mix64;

struct Rmat {
  uint32_t scale;
  uint64_t seed, mask;
  uint32_t cut[3];  // cumulative quadrant thresholds on a 32-bit uniform draw
  uint64_t mul[3], add[3];
  uint32_t shift;

  Rmat(uint32_t s, uint64_t sd) : scale(s), seed(sd) {
    const double two32 = 4294967296.0;
    cut[0] = (uint32_t)(0.57 * two32);
    cut[1] = (uint32_t)((0.57 + 0.19) * two32);
    cut[2] = (uint32_t)((0.57 + 0.19 + 0.19) * two32);
    mask = (1ull << s) - 1ull;
    for (uint64_t k = 0; k < 3; ++k) {
      mul[k] = mix64(sd ^ (0xA5A5ull + k)) | 1ull;
      add[k] = mix64(sd ^ (0x5A5Aull + k));
    }
    shift = s / 2 + 1;
  }

  uint64_t scatter(uint64_t x) const {
    for (int k = 0; k < 3; ++k) {
      x = (x * mul[k]) & mask;
      x ^= x >> shift;
      x = (x + add[k]) & mask;
    }
    return x;
  }

  void edge(uint64_t e, uint32_t* u, uint32_t* v) const {
    const uint64_t base = mix64(seed ^ mix64(e));
    uint64_t a = 0, b = 0;
    for (uint32_t level = 0; level < scale; ++level) {
      const uint64_t h = mix64(base + (level & ~1u));
      const uint32_t r = (uint32_t)(h >> (32 * (level & 1u)));
      const uint32_t q = r < cut[0] ? 0u : r < cut[1] ? 1u : r < cut[2] ? 2u : 3u;  // quadrant
      a = (a << 1) | (q >> 1);
      b = (b << 1) | (q & 1u);
    }
    *u = (uint32_t)scatter(a);
    *v = (uint32_t)scatter(b);
  }
};

int write_text(const std::string& name, const std::string& body) {
  FILE* f = fopen(name.c_str(), "w");
  if (!f) return 10;
  const size_t w = fwrite(body.data(), 1, body.size(), f);
  return (fclose(f) == 0 && w == body.size()) ? 0 : 10;
}

}  // namespace

extern "C" {

// RMAT CSR (source-major, sorted rows, no self loops or duplicates).  *off and *col are
// malloc'd; release them with oracle_host_free.  Returns 0, 9 (bad argument) or 12 (no memory).
int oracle_rmat(uint32_t scale, uint32_t edgefactor, uint64_t seed, int symmetric, uint64_t* n_out,
                uint64_t* m_out, uint64_t** off_out, uint32_t** col_out) {
  if (scale == 0 || scale > 31 || edgefactor == 0 || !n_out || !m_out || !off_out || !col_out) return 9;
  const Rmat gen(scale, seed);
  const uint64_t n = 1ull << scale, raw = (uint64_t)edgefactor << scale;
  std::vector<uint64_t> arcs;
  try {
    arcs.resize(symmetric ? 2 * raw : raw);
  } catch (...) {
    return 12;
  }
  uint64_t kept = 0;
#pragma omp parallel
  {
    std::vector<uint64_t> mine;
#pragma omp for schedule(static) nowait
    for (int64_t e = 0; e < (int64_t)raw; ++e) {
      uint32_t u, v;
      gen.edge((uint64_t)e, &u, &v);
      if (u == v) continue;
      mine.push_back(((uint64_t)u << 32) | v);
      if (symmetric) mine.push_back(((uint64_t)v << 32) | u);
    }
    uint64_t at;
#pragma omp atomic capture
    {
      at = kept;
      kept += mine.size();
    }
    std::copy(mine.begin(), mine.end(), arcs.begin() + at);
  }
  arcs.resize(kept);
  __gnu_parallel::sort(arcs.begin(), arcs.end());
  arcs.erase(std::unique(arcs.begin(), arcs.end()), arcs.end());
  const uint64_t m = arcs.size();
  uint64_t* off = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
  uint32_t* col = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  if (!off || !col) {
    free(off);
    free(col);
    return 12;
  }
  for (uint64_t i = 0; i < m; ++i) {
    off[(arcs[i] >> 32) + 1]++;
    col[i] = (uint32_t)arcs[i];
  }
  for (uint64_t v = 0; v < n; ++v) off[v + 1] += off[v];
  *n_out = n;
  *m_out = m;
  *off_out = off;
  *col_out = col;
  return 0;
}

void oracle_host_free(void* p) { free(p); }

// <prefix>.meta and <prefix>.edges.0 .. <prefix>.edges.<nfiles-1>; source u goes to file u % nfiles.
int oracle_write_edgelists(const char* prefix, uint64_t n, uint64_t m, const uint64_t* off, const uint32_t* col,
                           uint32_t nfiles) {
  if (!prefix || !off || nfiles == 0 || off[n] != m) return 9;
  int status = write_text(std::string(prefix) + ".meta", std::to_string(n) + " " + std::to_string(m) + "\n");
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t f = 0; f < (int64_t)nfiles; ++f) {
    std::string body;
    char line[48];
    for (uint64_t u = (uint64_t)f; u < n; u += nfiles)
      for (uint64_t a = off[u]; a < off[u + 1]; ++a) {
        const int k = snprintf(line, sizeof line, "%llu %u\n", (unsigned long long)u, col[a]);
        body.append(line, (size_t)k);
      }
    const int st = write_text(std::string(prefix) + ".edges." + std::to_string(f), body);
    if (st) {
#pragma omp atomic write
      status = st;
    }
  }
  return status;
}

// <prefix>.roots: the count, then one id per line.
int oracle_write_roots(const char* prefix, const uint32_t* roots, uint32_t count) {
  if (!prefix || (count && !roots)) return 9;
  std::string body = std::to_string(count) + "\n";
  for (uint32_t i = 0; i < count; ++i) body += std::to_string(roots[i]) + "\n";
  return write_text(std::string(prefix) + ".roots", body);
}

// The harness SSSP weight (1 + H(seed, min, max) % 255) of every arc of a CSR, in CSR order.
void oracle_sssp_weights_csr(uint64_t wseed, uint64_t n, const uint64_t* off, const uint32_t* col, uint32_t* w) {
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)n; ++u)
    for (uint64_t a = off[u]; a < off[u + 1]; ++a) w[a] = gre_oracle::sssp_weight(wseed, (uint64_t)u, col[a]);
}

}  // extern "C"
