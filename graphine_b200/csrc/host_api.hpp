// Internal host-side declarations shared by the C ABI translation units.
#pragma once
#include <stdint.h>

#include <vector>

namespace gre {

struct HostCSR {
  uint64_t n = 0, m = 0;
  std::vector<uint64_t> off;
  std::vector<uint32_t> col;
};

int host_rmat_csr(uint32_t scale, uint32_t edgefactor, uint64_t seed, int symmetric, HostCSR* out);
int host_write_edgelists(const char* prefix, uint64_t n, uint64_t m, const uint64_t* off,
                         const uint32_t* col, uint32_t nfiles);
int host_write_roots(const char* prefix, const uint32_t* roots, uint32_t count);
int host_read_roots(const char* prefix, std::vector<uint32_t>* roots);
void host_build_csr(uint64_t n, const std::vector<uint32_t>& src, const std::vector<uint32_t>& dst,
                    bool by_dst, std::vector<uint64_t>* off, std::vector<uint32_t>* col);
// the per-thread error text of the C ABI (graph.cu)
void set_error(const char* fmt, ...);
void clear_error();

}  // namespace gre
