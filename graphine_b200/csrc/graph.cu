// Graph handles: one device CSR (out-arcs) + CSC (in-arcs) per graph, uint32 ids, uint64
// offsets.  Replaces the reference's per-rank GraphInCSR + DistributedGraph id maps
// (Graph/LocalGraph.hpp:23-200, Graph/DistributedGraph.hpp:23-273): at one GPU every vertex is
// a master, so agents, scatter/combiner maps and hash indices disappear and lvid == vid.
//
// HBM layout per graph (n vertices, m arcs):
//   off[n+1] u64, col[m] u32                    CSR, source-major
//   roff[n+1] u64, rcol[m] u32, rarc[m] u64      CSC sorted by (dst, src, arc id) and the CSR
//                                                arc id of each CSC slot; aliased to the CSR
//                                                when the graph is symmetric (rarc on demand)
//   outdeg[n] u32 (indeg[n] u32)                 degrees
//   w32[m] u32 / w64[m] f64                      optional arc weights, CSR order
//   perm[n], iperm[n] u32, arc_rank[m] u32       relabelled graphs only: internal <-> caller
//                                                ids and each arc's caller position
#include <cub/cub.cuh>

#include <algorithm>
#include <mutex>
#include <vector>

#include "gre_internal.cuh"
#include "host_api.hpp"
#include "rmat.hpp"

namespace gre {

// ---------------------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------------------
static thread_local std::string t_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_error = buf;
}
void clear_error() { t_error.clear(); }
const char* last_error_text() { return t_error.c_str(); }

int cuda_status(cudaError_t e, const char* what, const char* file, int line) {
  set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // allocation failures are not sticky; clear them
    return GRE_OOM;
  }
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GRE_NO_DEVICE;
  return GRE_CUDA_ERROR;
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int num_sms() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

// The graph's stream is non-blocking: without a wait it would not be ordered after the caller's
// work on the legacy default stream (PyTorch's default stream; kernels and copies issued without
// a stream), and could read a device input before that work wrote it, or write a device output
// that work still reads.  Every call therefore starts by making the graph's stream wait for the
// legacy stream's work issued so far (an event, no host synchronisation).  Skipped while a stream
// capture is in progress (the legacy stream cannot be used then): a caller that captures, or that
// works on streams of its own, orders its buffers itself.
int use_graph(gre_graph g) {
  if (!g) {
    set_error("null graph handle");
    return GRE_NULL;
  }
  GRE_CUDA(cudaSetDevice(g->device));
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(g->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return GRE_SUCCESS;
  }
  if (cudaEventRecord(g->ev_caller, cudaStreamLegacy) != cudaSuccess) {  // another stream is being captured
    cudaGetLastError();
    return GRE_SUCCESS;
  }
  GRE_CUDA(cudaStreamWaitEvent(g->stream, g->ev_caller, 0));
  return GRE_SUCCESS;
}

int Workspace::get(int slot, size_t nbytes, void** out) {
  if (nbytes == 0) nbytes = 16;
  if (bytes[slot] < nbytes) {
    if (ptr[slot]) {
      cudaFree(ptr[slot]);
      ptr[slot] = nullptr;
      bytes[slot] = 0;
    }
    void* p = nullptr;
    GRE_CUDA(cudaMalloc(&p, nbytes));
    ptr[slot] = p;
    bytes[slot] = nbytes;
  }
  *out = ptr[slot];
  return GRE_SUCCESS;
}

void Workspace::release() {
  for (int i = 0; i < WS_NSLOTS; ++i) {
    if (ptr[i]) cudaFree(ptr[i]);
    ptr[i] = nullptr;
    bytes[i] = 0;
  }
}

// ---------------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------------
__global__ void k_degree(uint64_t n, const uint64_t* __restrict__ off, uint32_t* __restrict__ deg) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    deg[v] = (uint32_t)(off[v + 1] - off[v]);
}

// Row (source) of arc a by binary search over the offsets.
__device__ __forceinline__ uint32_t row_of_arc(const uint64_t* __restrict__ off, uint64_t n, uint64_t a) {
  uint64_t lo = 0, hi = n;  // find largest r with off[r] <= a
  while (hi - lo > 1) {
    const uint64_t mid = (lo + hi) >> 1;
    if (off[mid] <= a) lo = mid;
    else hi = mid;
  }
  return (uint32_t)lo;
}

__global__ void k_csc_keys(uint64_t n, uint64_t m, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                           uint64_t* __restrict__ keys, uint64_t* __restrict__ vals) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < m; a += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = row_of_arc(off, n, a);
    keys[a] = ((uint64_t)col[a] << 32) | u;
    vals[a] = a;
  }
}

__global__ void k_csc_split(uint64_t m, const uint64_t* __restrict__ keys, const uint64_t* __restrict__ vals,
                            uint32_t* __restrict__ rcol, uint64_t* __restrict__ rarc) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    rcol[i] = (uint32_t)(keys[i] & 0xffffffffull);
    if (rarc) rarc[i] = vals[i];
  }
}

// offsets[v] = first index i with (keys[i] >> 32) >= v, for v in [0, n]; keys sorted.
__global__ void k_offsets_from_sorted(uint64_t n, uint64_t m, const uint64_t* __restrict__ keys, uint64_t* __restrict__ off) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= n; v += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = m;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if ((keys[mid] >> 32) < v) lo = mid + 1;
      else hi = mid;
    }
    off[v] = lo;
  }
}

__global__ void k_rmat_keys(rmat::Params p, uint64_t m_raw, int symmetric, uint64_t self_key, uint64_t* __restrict__ keys) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m_raw; e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u, v;
    rmat::edge(p, e, &u, &v);
    const bool self = (u == v);
    keys[e] = self ? self_key : (((uint64_t)u << 32) | v);
    if (symmetric) keys[m_raw + e] = self ? self_key : (((uint64_t)v << 32) | u);
  }
}

__global__ void k_low32(uint64_t m, const uint64_t* __restrict__ keys, uint32_t* __restrict__ col) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
    col[i] = (uint32_t)(keys[i] & 0xffffffffull);
}

// weight of every arc from its endpoints' caller ids (perm maps internal -> caller ids)
__global__ void k_hash_weights(uint64_t n, uint64_t m, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                               const uint32_t* __restrict__ perm, uint64_t wseed, uint32_t* __restrict__ w) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < m; a += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = row_of_arc(off, n, a);
    const uint32_t v = col[a];
    w[a] = perm ? rmat::weight(wseed, perm[u], perm[v]) : rmat::weight(wseed, u, v);
  }
}

// relabelling: sort key = complement of the degree (decreasing degree, stable in id)
__global__ void k_reorder_keys(uint64_t n, const uint64_t* __restrict__ off, uint32_t* __restrict__ keys, uint32_t* __restrict__ ids) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t d = off[v + 1] - off[v];
    keys[v] = 0xffffffffu - (uint32_t)(d > 0xffffffffull ? 0xffffffffull : d);
    ids[v] = (uint32_t)v;
  }
}
__global__ void k_inverse_perm(uint64_t n, const uint32_t* __restrict__ perm, uint32_t* __restrict__ iperm) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    iperm[perm[i]] = (uint32_t)i;
}
// Relabelled arcs of caller row u (warp per row): key = new row << 32 | new column, value =
// the arc's position in its caller row.
__global__ void k_relabel_arcs(uint64_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                               const uint32_t* __restrict__ iperm, uint64_t* __restrict__ keys, uint32_t* __restrict__ rank) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t u = warp; u < n; u += nwarps) {
    const uint64_t a0 = off[u], len = off[u + 1] - a0;
    const uint64_t hi = (uint64_t)iperm[u] << 32;
    for (uint64_t k = lane; k < len; k += 32) {
      keys[a0 + k] = hi | iperm[col[a0 + k]];
      rank[a0 + k] = (uint32_t)k;
    }
  }
}

// out[a] = in[caller arc of internal arc a], the internal arcs sorted by (row, column) keys
template <class T>
__global__ void k_gather_by_rank(uint64_t m, const uint64_t* __restrict__ keys, const uint32_t* __restrict__ rank,
                                 const uint32_t* __restrict__ perm, const uint64_t* __restrict__ coff, const T* __restrict__ in,
                                 T* __restrict__ out) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < m; a += (uint64_t)gridDim.x * blockDim.x)
    out[a] = in[coff[perm[keys[a] >> 32]] + rank[a]];
}

__global__ void k_gather_f64(uint64_t m, const uint64_t* __restrict__ idx, const double* __restrict__ src, double* __restrict__ dst) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

__global__ void k_shift_u64(uint64_t cnt, const uint64_t* __restrict__ in, uint64_t add, uint64_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[i] + add;
}
__global__ void k_shift_u32(uint64_t cnt, const uint32_t* __restrict__ in, uint32_t add, uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[i] + add;
}

// ---------------------------------------------------------------------------------------------
// construction helpers
// ---------------------------------------------------------------------------------------------
int new_graph(int device, uint32_t flags, gre_graph* out) {
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device available");
    return GRE_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("device %d out of range (%d devices)", device, ndev);
    return GRE_INVALID_ARG;
  }
  GRE_CUDA(cudaSetDevice(device));
  gre_graph g = new gre_graph_s;
  g->device = device;
  g->flags = flags;
  cudaError_t e1 = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  cudaError_t e2 = cudaEventCreate(&g->ev0);
  cudaError_t e3 = cudaEventCreate(&g->ev1);
  if (e3 == cudaSuccess) e3 = cudaEventCreateWithFlags(&g->ev_caller, cudaEventDisableTiming);
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
    delete g;
    return cuda_status(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3), "stream/event create", __FILE__, __LINE__);
  }
  *out = g;
  return GRE_SUCCESS;
}

void destroy_graph(gre_graph g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  const bool sym_alias = (g->roff == g->off);
  cudaFree(g->off);
  cudaFree(g->col);
  if (!sym_alias) {
    cudaFree(g->roff);
    cudaFree(g->rcol);
  }
  cudaFree(g->rarc);
  if (g->indeg != g->outdeg) cudaFree(g->indeg);
  cudaFree(g->outdeg);
  cudaFree(g->w32);
  cudaFree(g->w64);
  cudaFree(g->rw64);
  free_bins(g->bins_in);
  free_bins(g->bins_out);
  free_bins(g->bins_sssp);
  cudaFree(g->bc_chunks.rows);
  cudaFree(g->bc_chunks.chunk_row);
  cudaFree(g->bc_chunks.chunk_begin);
  cudaFree(g->bc_chunks.first);
  cudaFree(g->bc_fpool);
  cudaFree(g->perm);
  cudaFree(g->iperm);
  cudaFree(g->arc_rank);
  g->sssp_split.release();
  g->ws.release();
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  if (g->ev_caller) cudaEventDestroy(g->ev_caller);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}


static int cub_temp(gre_graph g, size_t bytes, void** p) { return g->ws.get(WS_CUB, bytes, p); }

// CSC (in-arcs) from the CSR: sort (dst, src) keys with the arc id as value.
static int build_csc(gre_graph g) {
  const uint64_t n = g->n, m = g->m;
  GRE_CUDA(cudaMalloc(&g->roff, sizeof(uint64_t) * (n + 1)));
  GRE_CUDA(cudaMalloc(&g->rcol, sizeof(uint32_t) * (m ? m : 1)));
  GRE_CUDA(cudaMalloc(&g->rarc, sizeof(uint64_t) * (m ? m : 1)));
  if (m == 0) {
    GRE_CUDA(cudaMemsetAsync(g->roff, 0, sizeof(uint64_t) * (n + 1), g->stream));
    return GRE_SUCCESS;
  }
  uint64_t *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr;
  GRE_CUDA(cudaMalloc(&k0, sizeof(uint64_t) * m));
  cudaError_t e = cudaMalloc(&k1, sizeof(uint64_t) * m);
  if (e == cudaSuccess) e = cudaMalloc(&v0, sizeof(uint64_t) * m);
  if (e == cudaSuccess) e = cudaMalloc(&v1, sizeof(uint64_t) * m);
  int st = GRE_SUCCESS;
  if (e != cudaSuccess) st = cuda_status(e, "cudaMalloc (CSC build)", __FILE__, __LINE__);
  if (!st) {
    k_csc_keys<<<grid_for(m, 256), 256, 0, g->stream>>>(n, m, g->off, g->col, k0, v0);
    cub::DoubleBuffer<uint64_t> dk(k0, k1), dv(v0, v1);
    int bits = 1;
    while (bits < 32 && (1ull << bits) < n) ++bits;
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, m, 0, 32 + bits, g->stream);
    void* tmp = nullptr;
    st = cub_temp(g, tb, &tmp);
    if (!st) {
      e = cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dv, m, 0, 32 + bits, g->stream);
      if (e != cudaSuccess) st = cuda_status(e, "SortPairs", __FILE__, __LINE__);
    }
    if (!st) {
      k_csc_split<<<grid_for(m, 256), 256, 0, g->stream>>>(m, dk.Current(), dv.Current(), g->rcol, g->rarc);
      k_offsets_from_sorted<<<grid_for(n + 1, 256), 256, 0, g->stream>>>(n, m, dk.Current(), g->roff);
      e = cudaStreamSynchronize(g->stream);
      if (e != cudaSuccess) st = cuda_status(e, "CSC build", __FILE__, __LINE__);
    }
  }
  cudaFree(k0);
  cudaFree(k1);
  cudaFree(v0);
  cudaFree(v1);
  return st;
}

// Degrees, maxima and the CSC; called once the CSR is on the device.
// warp per row: clears *sorted if a row's columns decrease somewhere
__global__ void k_rows_sorted(uint64_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                              unsigned int* __restrict__ sorted) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  bool ok = true;
  for (uint64_t v = warp; v < n; v += nwarps)
    for (uint64_t a = off[v] + lane; a + 1 < off[v + 1]; a += 32) ok = ok && col[a] <= col[a + 1];
  if (!__all_sync(0xffffffffu, ok) && lane == 0) atomicAnd(sorted, 0u);
}

int finish_graph(gre_graph g) {
  const uint64_t n = g->n;
  {
    unsigned int* flag = nullptr;
    GRE_CHECK(g->ws.get(WS_COUNTERS, 64, (void**)&flag));
    const unsigned int one = 1;
    GRE_CUDA(cudaMemcpyAsync(flag, &one, sizeof one, cudaMemcpyHostToDevice, g->stream));
    k_rows_sorted<<<grid_for(n * 32, 256), 256, 0, g->stream>>>(n, g->off, g->col, flag);
    GRE_LAUNCH_CHECK();
    unsigned int h = 0;
    GRE_CUDA(cudaMemcpyAsync(&h, flag, sizeof h, cudaMemcpyDeviceToHost, g->stream));
    GRE_CUDA(cudaStreamSynchronize(g->stream));
    g->csr_sorted = h != 0;
  }
  GRE_CUDA(cudaMalloc(&g->outdeg, sizeof(uint32_t) * n));
  k_degree<<<grid_for(n, 256), 256, 0, g->stream>>>(n, g->off, g->outdeg);
  GRE_LAUNCH_CHECK();
  if (g->symmetric()) {
    g->roff = g->off;
    g->rcol = g->col;
    g->indeg = g->outdeg;
  } else {
    GRE_CHECK(build_csc(g));
    GRE_CUDA(cudaMalloc(&g->indeg, sizeof(uint32_t) * n));
    k_degree<<<grid_for(n, 256), 256, 0, g->stream>>>(n, g->roff, g->indeg);
    GRE_LAUNCH_CHECK();
  }
  // maxima (host side, one pass over the degree arrays)
  size_t tb = 0;
  uint32_t* dmax = nullptr;
  void* tmp = nullptr;
  GRE_CHECK(g->ws.get(WS_COUNTERS, 64, (void**)&dmax));
  cub::DeviceReduce::Max(nullptr, tb, g->outdeg, dmax, n, g->stream);
  GRE_CHECK(cub_temp(g, tb, &tmp));
  GRE_CUDA(cub::DeviceReduce::Max(tmp, tb, g->outdeg, dmax, n, g->stream));
  GRE_CUDA(cub::DeviceReduce::Max(tmp, tb, g->indeg, dmax + 1, n, g->stream));
  uint32_t hm[2] = {0, 0};
  GRE_CUDA(cudaMemcpyAsync(hm, dmax, sizeof hm, cudaMemcpyDeviceToHost, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  g->max_outdeg = hm[0];
  g->max_indeg = hm[1];
  return GRE_SUCCESS;
}

// Drops everything derived from the CSR (degrees, CSC, arc maps, bins, chunk tables).
static void drop_derived(gre_graph g) {
  g->sssp_split.release();
  const bool alias = (g->roff == g->off);
  if (!alias) {
    cudaFree(g->roff);
    cudaFree(g->rcol);
  }
  g->roff = nullptr;
  g->rcol = nullptr;
  cudaFree(g->rarc);
  g->rarc = nullptr;
  cudaFree(g->rw64);
  g->rw64 = nullptr;
  if (g->indeg != g->outdeg) cudaFree(g->indeg);
  cudaFree(g->outdeg);
  g->indeg = g->outdeg = nullptr;
  free_bins(g->bins_in);
  free_bins(g->bins_out);
  free_bins(g->bins_sssp);
  cudaFree(g->bc_chunks.rows);
  cudaFree(g->bc_chunks.chunk_row);
  cudaFree(g->bc_chunks.chunk_begin);
  cudaFree(g->bc_chunks.first);
  g->bc_chunks = ChunkTable();
}

// Relabel by decreasing degree: new row i = old row perm[i], neighbour ids mapped through
// iperm, and each row's arcs sorted by new neighbour id (a stable sort: parallel arcs keep their
// caller order).  Sorted rows put the arcs towards hubs (small new ids) side by side, so the
// gathers of a warp share more cache lines.  Weights move with their arcs; arc_rank keeps each
// arc's caller position for per-arc inputs and outputs.
int reorder_graph(gre_graph g) {
  if (g->perm) return GRE_SUCCESS;  // already relabelled
  const uint64_t n = g->n, m = g->m;
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  uint32_t *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr, *perm = nullptr, *iperm = nullptr;
  uint64_t *ak0 = nullptr, *ak1 = nullptr, *noff = nullptr;
  uint32_t *av0 = nullptr, *av1 = nullptr, *rank = nullptr;
  uint32_t* ncol = nullptr;
  uint32_t* nw32 = nullptr;
  double* nw64 = nullptr;
  auto free_sort = [&]() {
    cudaFree(k0);
    cudaFree(k1);
    cudaFree(v0);
    cudaFree(v1);
    cudaFree(ak0);
    cudaFree(ak1);
    k0 = k1 = v0 = v1 = nullptr;
    ak0 = ak1 = nullptr;
  };
  const uint64_t mm = m ? m : 1;
  cudaError_t e = cudaMalloc(&k0, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&k1, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&v0, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&v1, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&iperm, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&ak0, 8 * mm);
  if (e == cudaSuccess) e = cudaMalloc(&ak1, 8 * mm);
  if (e == cudaSuccess) e = cudaMalloc(&av0, 4 * mm);
  if (e == cudaSuccess) e = cudaMalloc(&av1, 4 * mm);
  if (e == cudaSuccess) e = cudaMalloc(&noff, 8 * (n + 1));
  if (e == cudaSuccess) e = cudaMalloc(&ncol, 4 * mm);
  if (e == cudaSuccess && g->w32) e = cudaMalloc(&nw32, 4 * mm);
  if (e == cudaSuccess && g->w64) e = cudaMalloc(&nw64, 8 * mm);
  int st = e == cudaSuccess ? GRE_SUCCESS : cuda_status(e, "cudaMalloc (reorder)", __FILE__, __LINE__);
  if (!st) {
    // vertex order: stable sort by decreasing degree
    k_reorder_keys<<<grid_for(n, 256), 256, 0, g->stream>>>(n, g->off, k0, v0);
    cub::DoubleBuffer<uint32_t> dk(k0, k1), dv(v0, v1);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, n, 0, 32, g->stream);
    void* tmp = nullptr;
    st = cub_temp(g, tb, &tmp);
    if (!st) {
      e = cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dv, n, 0, 32, g->stream);
      if (e != cudaSuccess) st = cuda_status(e, "SortPairs (reorder)", __FILE__, __LINE__);
    }
    if (!st) {
      perm = dv.Current();
      k_inverse_perm<<<grid_for(n, 256), 256, 0, g->stream>>>(n, perm, iperm);
    }
  }
  if (!st && m) {
    // arcs: sort (new row, new column) keys carrying each arc's caller position
    k_relabel_arcs<<<grid_for(n * 32, 256), 256, 0, g->stream>>>(n, g->off, g->col, iperm, ak0, av0);
    int bits = 1;
    while (bits < 32 && (1ull << bits) < n) ++bits;
    cub::DoubleBuffer<uint64_t> dk(ak0, ak1);
    cub::DoubleBuffer<uint32_t> dv(av0, av1);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, m, 0, 32 + bits, g->stream);
    void* tmp = nullptr;
    st = cub_temp(g, tb, &tmp);
    if (!st) {
      e = cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dv, m, 0, 32 + bits, g->stream);
      if (e != cudaSuccess) st = cuda_status(e, "SortPairs (reorder arcs)", __FILE__, __LINE__);
    }
    if (!st) {
      const uint64_t* keys = dk.Current();
      rank = dv.Current();
      k_low32<<<grid_for(m, 256), 256, 0, g->stream>>>(m, keys, ncol);
      k_offsets_from_sorted<<<grid_for(n + 1, 256), 256, 0, g->stream>>>(n, m, keys, noff);
      if (nw32) k_gather_by_rank<uint32_t><<<grid_for(m, 256), 256, 0, g->stream>>>(m, keys, rank, perm, g->off, g->w32, nw32);
      if (nw64) k_gather_by_rank<double><<<grid_for(m, 256), 256, 0, g->stream>>>(m, keys, rank, perm, g->off, g->w64, nw64);
    }
  } else if (!st) {
    GRE_CUDA(cudaMemsetAsync(noff, 0, 8 * (n + 1), g->stream));
  }
  if (!st) {
    e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) st = cuda_status(e, "reorder", __FILE__, __LINE__);
  }
  if (st) {
    free_sort();
    cudaFree(av0);
    cudaFree(av1);
    cudaFree(iperm);
    cudaFree(noff);
    cudaFree(ncol);
    cudaFree(nw32);
    cudaFree(nw64);
    return st;
  }
  // keep the sorted vertex ids as perm and the sorted ranks as arc_rank; release the rest
  if (perm == v0) v0 = nullptr;
  else v1 = nullptr;
  if (rank == av0) av0 = nullptr;
  else if (rank == av1) av1 = nullptr;
  free_sort();
  cudaFree(av0);
  cudaFree(av1);
  drop_derived(g);
  cudaFree(g->off);
  cudaFree(g->col);
  cudaFree(g->w32);
  cudaFree(g->w64);
  g->off = noff;
  g->col = ncol;
  g->w32 = nw32;
  g->w64 = nw64;
  g->perm = perm;
  g->iperm = iperm;
  g->arc_rank = rank;
  g->h_iperm.resize(n);
  GRE_CUDA(cudaMemcpy(g->h_iperm.data(), iperm, 4 * n, cudaMemcpyDeviceToHost));
  g->flags |= GRE_GRAPH_REORDER;
  return GRE_SUCCESS;
}

static int validate_csr_host(uint64_t n, uint64_t m, const uint64_t* off, const uint32_t* col) {
  if (off[0] != 0 || off[n] != m) {
    set_error("row offsets must start at 0 and end at m");
    return GRE_INVALID_ARG;
  }
  for (uint64_t v = 0; v < n; ++v)
    if (off[v + 1] < off[v]) {
      set_error("row offsets decrease at %llu", (unsigned long long)v);
      return GRE_INVALID_ARG;
    }
  for (uint64_t a = 0; a < m; ++a)
    if (col[a] >= n) {
      set_error("arc %llu: vertex id %u >= n = %llu", (unsigned long long)a, col[a], (unsigned long long)n);
      return GRE_INVALID_ARG;
    }
  return GRE_SUCCESS;
}

static int make_from_host_csr(uint64_t n, uint64_t m, const uint64_t* off, const uint32_t* col, uint32_t flags,
                              int device, gre_graph* out) {
  GRE_CHECK(validate_csr_host(n, m, off, col));
  gre_graph g = nullptr;
  GRE_CHECK(new_graph(device, flags, &g));
  GraphGuard guard{g};
  g->n = n;
  g->m = m;
  GRE_CUDA(cudaMalloc(&g->off, sizeof(uint64_t) * (n + 1)));
  GRE_CUDA(cudaMalloc(&g->col, sizeof(uint32_t) * (m ? m : 1)));
  GRE_CUDA(cudaMemcpyAsync(g->off, off, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, g->stream));
  if (m) GRE_CUDA(cudaMemcpyAsync(g->col, col, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, g->stream));
  if (flags & GRE_GRAPH_REORDER) GRE_CHECK(reorder_graph(g));
  GRE_CHECK(finish_graph(g));
  *out = guard.release();
  return GRE_SUCCESS;
}

// Relabel an existing graph and rebuild what depends on the CSR.
static int reorder_existing(gre_graph g) {
  if (g->perm) return GRE_SUCCESS;
  GRE_CHECK(reorder_graph(g));
  GRE_CHECK(finish_graph(g));
  if (g->w64) {
    GRE_CHECK(ensure_rarc(g));
    GRE_CUDA(cudaMalloc(&g->rw64, sizeof(double) * (g->m ? g->m : 1)));
    if (g->m) k_gather_f64<<<grid_for(g->m, 256), 256, 0, g->stream>>>(g->m, g->rarc, g->w64, g->rw64);
    GRE_LAUNCH_CHECK();
  }
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  return GRE_SUCCESS;
}

int ensure_rarc(gre_graph g) {
  if (g->rarc) return GRE_SUCCESS;
  // symmetric alias: build a true CSC with its arc map and stop aliasing
  g->roff = nullptr;
  g->rcol = nullptr;
  int st = build_csc(g);
  if (st) {
    cudaFree(g->roff);
    cudaFree(g->rcol);
    cudaFree(g->rarc);
    g->roff = g->off;
    g->rcol = g->col;
    g->rarc = nullptr;
  }
  return st;
}

}  // namespace gre

using namespace gre;

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

const char* gre_status_str(int s) {
  static const char* words[] = {"success", "failure", "no_buffer", "null", "finished", "unfinished",
                                "initialized", "uninitialized", "not_implemented", "invalid_argument",
                                "io_error", "cuda_error", "out_of_memory", "timeout", "no_device"};
  if (s < 0 || s > GRE_NO_DEVICE) return "unknown_status";
  return words[s];
}

const char* gre_last_error(void) { return last_error_text(); }

int gre_device_count(int* count) {
  if (!count) return GRE_NULL;
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    c = 0;
  }
  *count = c;
  return GRE_SUCCESS;
}

int gre_graph_load(const char* prefix, uint32_t flags, int device, gre_graph* out) {
  if (!prefix || !out) return GRE_NULL;
  clear_error();
  return device_ingest(prefix, flags, device, out);
}

int gre_graph_load_parts(const char* prefix, uint32_t nparts, uint32_t flags, int device, gre_graph* out) {
  if (!prefix || !out) return GRE_NULL;
  clear_error();
  return device_ingest_parts(prefix, nparts, flags, device, out);
}

int gre_graph_from_edges(uint64_t n, uint64_t m, const uint32_t* src, const uint32_t* dst, uint32_t flags, int device,
                         gre_graph* out) {
  if (!out || (m && (!src || !dst))) return GRE_NULL;
  if (n == 0 || n > 0xffffffffull) return GRE_INVALID_ARG;
  clear_error();
  std::vector<uint32_t> s(src, src + m), d(dst, dst + m);
  for (uint64_t i = 0; i < m; ++i)
    if (s[i] >= n || d[i] >= n) {
      set_error("edge %llu has a vertex id >= n", (unsigned long long)i);
      return GRE_INVALID_ARG;
    }
  std::vector<uint64_t> off;
  std::vector<uint32_t> col;
  host_build_csr(n, s, d, false, &off, &col);
  return make_from_host_csr(n, m, off.data(), col.data(), flags, device, out);
}

int gre_graph_from_csr(uint64_t n, uint64_t m, const uint64_t* row_off, const uint32_t* col, uint32_t flags, int device,
                       gre_graph* out) {
  if (!out || !row_off || (m && !col)) return GRE_NULL;
  if (n == 0 || n > 0xffffffffull) return GRE_INVALID_ARG;
  clear_error();
  if (!is_device_ptr(row_off) && !is_device_ptr(col)) return make_from_host_csr(n, m, row_off, col, flags, device, out);
  // device arrays: copy back for validation, then build as from the host
  std::vector<uint64_t> off(n + 1);
  std::vector<uint32_t> c(m);
  GRE_CUDA(cudaMemcpy(off.data(), row_off, sizeof(uint64_t) * (n + 1), cudaMemcpyDefault));
  if (m) GRE_CUDA(cudaMemcpy(c.data(), col, sizeof(uint32_t) * m, cudaMemcpyDefault));
  return make_from_host_csr(n, m, off.data(), c.data(), flags, device, out);
}

int gre_graph_rmat(uint32_t scale, uint32_t edgefactor, uint64_t seed, int symmetric, int device, gre_graph* out) {
  if (!out) return GRE_NULL;
  if (scale == 0 || scale > 31 || edgefactor == 0) return GRE_INVALID_ARG;
  clear_error();
  gre_graph g = nullptr;
  GRE_CHECK(new_graph(device, (symmetric ? (GRE_DIR_INOUT | GRE_GRAPH_SYMMETRIC) : GRE_DIR_OUT), &g));
  GraphGuard guard{g};
  const rmat::Params p = rmat::make_params(scale, seed);
  const uint64_t n = 1ull << scale;
  const uint64_t m_raw = (uint64_t)edgefactor << scale;
  const uint64_t nk = symmetric ? 2 * m_raw : m_raw;
  const uint64_t self_key = n << 32;  // sorts after every real arc
  uint64_t *k0 = nullptr, *k1 = nullptr, *nsel = nullptr;
  GRE_CUDA(cudaMalloc(&k0, sizeof(uint64_t) * nk));
  cudaError_t e = cudaMalloc(&k1, sizeof(uint64_t) * nk);
  if (e == cudaSuccess) e = cudaMalloc(&nsel, sizeof(uint64_t));
  int st = e == cudaSuccess ? GRE_SUCCESS : cuda_status(e, "cudaMalloc (rmat keys)", __FILE__, __LINE__);
  uint64_t m = 0;
  uint64_t* uniq = nullptr;
  if (!st) {
    k_rmat_keys<<<grid_for(m_raw, 256), 256, 0, g->stream>>>(p, m_raw, symmetric, self_key, k0);
    cub::DoubleBuffer<uint64_t> dk(k0, k1);
    size_t tb = 0;
    const int end_bit = 32 + (int)scale + 1;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, dk, nk, 0, end_bit, g->stream);
    void* tmp = nullptr;
    st = cub_temp(g, tb, &tmp);
    if (!st) {
      e = cub::DeviceRadixSort::SortKeys(tmp, tb, dk, nk, 0, end_bit, g->stream);
      if (e != cudaSuccess) st = cuda_status(e, "SortKeys (rmat)", __FILE__, __LINE__);
    }
    if (!st) {
      uint64_t* in = dk.Current();
      uniq = dk.Alternate();
      tb = 0;
      cub::DeviceSelect::Unique(nullptr, tb, in, uniq, nsel, nk, g->stream);
      st = cub_temp(g, tb, &tmp);
      if (!st) {
        e = cub::DeviceSelect::Unique(tmp, tb, in, uniq, nsel, nk, g->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&m, nsel, sizeof m, cudaMemcpyDeviceToHost, g->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
        if (e != cudaSuccess) st = cuda_status(e, "Unique (rmat)", __FILE__, __LINE__);
      }
    }
    if (!st) {
      uint64_t last = 0;
      if (m) {
        e = cudaMemcpy(&last, uniq + m - 1, sizeof last, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = cuda_status(e, "rmat tail", __FILE__, __LINE__);
        if (last == self_key) --m;
      }
    }
    if (!st) {
      g->n = n;
      g->m = m;
      e = cudaMalloc(&g->off, sizeof(uint64_t) * (n + 1));
      if (e == cudaSuccess) e = cudaMalloc(&g->col, sizeof(uint32_t) * (m ? m : 1));
      if (e != cudaSuccess) st = cuda_status(e, "cudaMalloc (rmat csr)", __FILE__, __LINE__);
    }
    if (!st) {
      k_low32<<<grid_for(m, 256), 256, 0, g->stream>>>(m, uniq, g->col);
      k_offsets_from_sorted<<<grid_for(n + 1, 256), 256, 0, g->stream>>>(n, m, uniq, g->off);
      e = cudaStreamSynchronize(g->stream);
      if (e != cudaSuccess) st = cuda_status(e, "rmat csr", __FILE__, __LINE__);
    }
  }
  cudaFree(k0);
  cudaFree(k1);
  cudaFree(nsel);
  if (st) return st;
  GRE_CHECK(finish_graph(g));
  *out = guard.release();
  return GRE_SUCCESS;
}

int gre_graph_union(const gre_graph* graphs, uint32_t k, int device, gre_graph* out, uint64_t* vertex_offset) {
  if (!graphs || !out || !vertex_offset || k == 0) return GRE_NULL;
  clear_error();
  uint64_t n = 0, m = 0;
  bool sym = true, all_w32 = true, w32_sym = true;
  for (uint32_t i = 0; i < k; ++i) {
    if (!graphs[i]) return GRE_NULL;
    if (graphs[i]->perm) {
      set_error("gre_graph_union: member %u is relabelled; build the union from unrelabelled graphs", i);
      return GRE_INVALID_ARG;
    }
    vertex_offset[i] = n;
    n += graphs[i]->n;
    m += graphs[i]->m;
    sym = sym && graphs[i]->symmetric();
    all_w32 = all_w32 && graphs[i]->w32;
    w32_sym = w32_sym && graphs[i]->w32_symmetric;
  }
  vertex_offset[k] = n;
  if (n > 0xffffffffull) return GRE_INVALID_ARG;
  gre_graph g = nullptr;
  GRE_CHECK(new_graph(device, sym ? (GRE_DIR_INOUT | GRE_GRAPH_SYMMETRIC) : GRE_DIR_INOUT, &g));
  GraphGuard guard{g};
  g->n = n;
  g->m = m;
  GRE_CUDA(cudaMalloc(&g->off, sizeof(uint64_t) * (n + 1)));
  GRE_CUDA(cudaMalloc(&g->col, sizeof(uint32_t) * (m ? m : 1)));
  if (all_w32) GRE_CUDA(cudaMalloc(&g->w32, sizeof(uint32_t) * (m ? m : 1)));
  g->w32_symmetric = all_w32 && w32_sym && sym;
  uint64_t vb = 0, ab = 0;
  for (uint32_t i = 0; i < k; ++i) {
    gre_graph s = graphs[i];
    GRE_CUDA(cudaStreamSynchronize(s->stream));
    k_shift_u64<<<grid_for(s->n, 256), 256, 0, g->stream>>>(s->n, s->off, ab, g->off + vb);
    k_shift_u32<<<grid_for(s->m, 256), 256, 0, g->stream>>>(s->m, s->col, (uint32_t)vb, g->col + ab);
    if (all_w32 && s->m)
      GRE_CUDA(cudaMemcpyAsync(g->w32 + ab, s->w32, sizeof(uint32_t) * s->m, cudaMemcpyDeviceToDevice, g->stream));
    vb += s->n;
    ab += s->m;
  }
  GRE_CUDA(cudaMemcpyAsync(g->off + n, &m, sizeof(uint64_t), cudaMemcpyHostToDevice, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  GRE_CHECK(finish_graph(g));
  *out = guard.release();
  return GRE_SUCCESS;
}

int gre_graph_free(gre_graph g) {
  if (!g) return GRE_NULL;
  destroy_graph(g);
  return GRE_SUCCESS;
}

int gre_graph_info(gre_graph g, uint64_t* n, uint64_t* m, uint32_t* flags) {
  if (!g) return GRE_NULL;
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (flags) *flags = g->flags;
  return GRE_SUCCESS;
}

int gre_graph_reorder(gre_graph g) {
  if (!g) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  return reorder_existing(g);
}

int gre_graph_outdegree(gre_graph g, uint32_t* outdeg) {
  if (!g || !outdeg) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  uint32_t* dout = nullptr;
  GRE_CHECK(prepare_output(g, outdeg, g->n, WS_OUTBUF, &dout));
  if (g->perm) GRE_CHECK(perm_out_end(g, g->outdeg, dout, 1, 4));
  else GRE_CUDA(cudaMemcpyAsync(dout, g->outdeg, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToDevice, g->stream));
  GRE_CHECK(finish_output(g, outdeg, dout, g->n));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  return GRE_SUCCESS;
}

int gre_graph_csr(gre_graph g, uint64_t* row_off, uint32_t* col) {
  if (!g || !row_off || (g->m && !col)) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  if (g->perm) return caller_csr(g, row_off, col);
  GRE_CUDA(cudaMemcpyAsync(row_off, g->off, sizeof(uint64_t) * (g->n + 1), cudaMemcpyDefault, g->stream));
  if (g->m) GRE_CUDA(cudaMemcpyAsync(col, g->col, sizeof(uint32_t) * g->m, cudaMemcpyDefault, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  return GRE_SUCCESS;
}

// Per-arc input in the arc order of gre_graph_csr -> device array in internal arc order.
static int upload_arcs(gre_graph g, const void* w, size_t elem, void* dst) {
  if (!g->m) return GRE_SUCCESS;
  const void* src = w;
  if (!is_device_ptr(w)) {
    void* tmp = nullptr;
    GRE_CHECK(g->ws.get(WS_PERM_IN, elem * g->m, &tmp));
    GRE_CUDA(cudaMemcpyAsync(tmp, w, elem * g->m, cudaMemcpyHostToDevice, g->stream));
    src = tmp;
  }
  return arcs_to_internal(g, src, dst, elem);
}

int gre_graph_set_weights_u32(gre_graph g, const uint32_t* w) {
  if (!g || (g->m && !w)) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  if (!g->w32) GRE_CUDA(cudaMalloc(&g->w32, sizeof(uint32_t) * (g->m ? g->m : 1)));
  GRE_CHECK(upload_arcs(g, w, 4, g->w32));
  g->w32_mean = -1.0;
  g->w32_symmetric = false;  // explicit per-arc weights: not known to be symmetric
  g->sssp_split.release();
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  return GRE_SUCCESS;
}

int gre_graph_set_weights_hash(gre_graph g, uint64_t wseed) {
  if (!g) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  if (!g->w32) GRE_CUDA(cudaMalloc(&g->w32, sizeof(uint32_t) * (g->m ? g->m : 1)));
  if (g->m) k_hash_weights<<<grid_for(g->m, 256), 256, 0, g->stream>>>(g->n, g->m, g->off, g->col, g->perm, wseed, g->w32);
  GRE_LAUNCH_CHECK();
  g->w32_mean = -1.0;
  g->w32_symmetric = g->symmetric();  // a function of the undirected edge
  g->sssp_split.release();
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  return GRE_SUCCESS;
}

int gre_graph_set_weights_f64(gre_graph g, const double* w) {
  if (!g || (g->m && !w)) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  if (!g->w64) GRE_CUDA(cudaMalloc(&g->w64, sizeof(double) * (g->m ? g->m : 1)));
  GRE_CHECK(upload_arcs(g, w, 8, g->w64));
  GRE_CHECK(ensure_rarc(g));
  if (!g->rw64) GRE_CUDA(cudaMalloc(&g->rw64, sizeof(double) * (g->m ? g->m : 1)));
  if (g->m) k_gather_f64<<<grid_for(g->m, 256), 256, 0, g->stream>>>(g->m, g->rarc, g->w64, g->rw64);
  GRE_LAUNCH_CHECK();
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  return GRE_SUCCESS;
}

}  // extern "C"
