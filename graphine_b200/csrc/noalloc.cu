// gre_bfs_noalloc: direction-optimising BFS that allocates no memory.
//
// Some callers cannot let a library allocate device memory: a serving process whose device
// memory is reserved up front and capped by its own pool allocator (a cudaMalloc outside the
// pool fails or breaks its budget), or a latency-critical loop that cannot afford the implicit
// device synchronisation of cudaMalloc / cudaFree.  For them this entry point keeps its scratch
// (frontier queues and bitmaps, the degree scan, counters, the scan's temporary storage) in one
// file-scope __device__ array of kNoAllocScratchBytes, and takes a device buffer for its result.
// The graph itself is an input the caller created beforehand.
//
// The array is shared by every call on a device and keeps the last call's contents: everything
// that must start at zero is cleared at the start of each call, and calls that overlap on the
// GPU (two streams, two threads) race on it.  The device address of the array is looked up once
// per device, with that device current, by the first call on it (cudaGetSymbolAddress), and again
// if that device's context was replaced since (cudaDeviceReset); make the first call after such
// a change before any stream capture.  Every GPU that loads this library's module holds the
// array until the process exits.
//
// It launches the kernels of the workspace-backed gre_bfs (bfs.cu) with pointers carved from the
// array, so both compute the same levels.
#include <cub/cub.cuh>

#include <algorithm>
#include <mutex>

#include "gre_internal.cuh"

namespace gre {

struct BfsCounters {
  unsigned long long next_count;
  unsigned long long next_arcs;
  unsigned long long scanned;
  unsigned long long pad;
};

// kernels defined in bfs.cu
__global__ void k_bfs_seed(const uint32_t* __restrict__ roots, uint32_t nroots, int32_t* __restrict__ level,
                           uint32_t* __restrict__ vis, uint32_t* __restrict__ queue, const uint64_t* __restrict__ off,
                           BfsCounters* __restrict__ c);
__global__ void k_frontier_degrees(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ off,
                                   uint64_t* __restrict__ deg);
__global__ void __launch_bounds__(256) k_td_expand(const uint32_t* __restrict__ queue, uint64_t nq, const uint64_t* __restrict__ prefix,
                                                   uint64_t total, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                   uint32_t* __restrict__ vis, int32_t* __restrict__ level, int32_t next_level,
                                                   uint32_t* __restrict__ next_queue, BfsCounters* __restrict__ c);
__global__ void k_queue_to_bits(const uint32_t* __restrict__ queue, uint64_t nq, uint32_t* __restrict__ bits);
__global__ void __launch_bounds__(256) k_bu_step(uint64_t n, const uint64_t* __restrict__ roff, const uint32_t* __restrict__ rcol,
                                                 const uint64_t* __restrict__ off, const uint32_t* __restrict__ front,
                                                 uint32_t* __restrict__ next, uint32_t* __restrict__ vis, int32_t* __restrict__ level,
                                                 int32_t next_level, BfsCounters* __restrict__ c);
__global__ void k_bits_to_queue(uint64_t n, const uint32_t* __restrict__ bits, uint32_t* __restrict__ queue,
                                unsigned long long* __restrict__ count);

constexpr uint64_t kNoAllocScratchBytes = 32ull << 20;  // 32 MiB
constexpr uint64_t kNoAllocMaxVertices = 1ull << 20;    // graphs of up to 1,048,576 vertices

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// caller order of the internal levels (relabelled graphs)
__global__ void k_noalloc_unperm(uint64_t n, const uint32_t* __restrict__ iperm, const int32_t* __restrict__ in,
                                 int32_t* __restrict__ out) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    out[v] = in[iperm[v]];
}

static std::mutex g_scratch_mu;
static void* g_scratch_addr[256];
static void* g_scratch_ctx[256];  // the context the address was looked up in

// The current context, through the driver entry point the runtime exposes (no libcuda link).
typedef int (*CtxGetCurrentFn)(void**);
static void* current_context() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return (CtxGetCurrentFn)f;
  }();
  void* ctx = nullptr;
  if (fn) fn(&ctx);
  return ctx;
}

// Device address of the scratch array on `device` (that device current).  Looked up once per
// device, and again only if the device's context changed since (after a cudaDeviceReset the
// module, and with it the array, is loaded anew at another address).
static int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= 256) return GRE_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  void* ctx = current_context();
  if (!g_scratch_addr[device] || ctx != g_scratch_ctx[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    g_scratch_addr[device] = p;
    g_scratch_ctx[device] = ctx;
  }
  *out = (unsigned char*)g_scratch_addr[device];
  return GRE_SUCCESS;
}

// `p` is device memory that the graph's device can write: memory of that device, or managed.
static bool on_device(const void* p, int device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the sticky-free error of an unregistered host pointer
    return false;
  }
  return a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == device);
}

static uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }

}  // namespace gre

using namespace gre;

extern "C" {

int gre_bfs_noalloc(gre_graph g, uint32_t src, int32_t* level, gre_stats* st) {
  if (!g || !level) return GRE_NULL;
  const uint64_t n = g->n;
  if (n > kNoAllocMaxVertices) {
    set_error("gre_bfs_noalloc: %llu vertices exceed the %llu this entry point's fixed scratch serves; use gre_bfs",
              (unsigned long long)n, (unsigned long long)kNoAllocMaxVertices);
    return GRE_INVALID_ARG;
  }
  if (src >= n) {
    set_error("gre_bfs_noalloc: source %u >= n", src);
    return GRE_INVALID_ARG;
  }
  GRE_CHECK(use_graph(g));
  if (!on_device(level, g->device)) {
    set_error("gre_bfs_noalloc: `level` must be device memory on the graph's device %d (this entry point "
              "stages nothing)", g->device);
    return GRE_INVALID_ARG;
  }
  unsigned char* base = nullptr;
  GRE_CHECK(scratch_address(g->device, &base));
  stats_reset(st);

  // carve the scratch
  const uint64_t nwords = (n + 31) >> 5;
  uint64_t o = 0;
  auto carve = [&](uint64_t bytes) {
    unsigned char* p = base + o;
    o = align256(o + bytes);
    return (void*)p;
  };
  uint32_t* vis = (uint32_t*)carve(4 * nwords);
  uint32_t* qa = (uint32_t*)carve(4 * n);
  uint32_t* qb = (uint32_t*)carve(4 * n);
  uint32_t* bits_a = (uint32_t*)carve(4 * nwords);
  uint32_t* bits_b = (uint32_t*)carve(4 * nwords);
  uint64_t* deg = (uint64_t*)carve(8 * (n + 1));
  uint64_t* prefix = (uint64_t*)carve(8 * (n + 1));
  BfsCounters* c = (BfsCounters*)carve(sizeof(BfsCounters));
  uint32_t* droot = (uint32_t*)carve(4);
  int32_t* lv = g->perm ? (int32_t*)carve(4 * n) : level;
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, deg, prefix, n + 1, g->stream);
  void* cub_tmp = carve(cub_bytes);
  if (o > kNoAllocScratchBytes) {
    set_error("gre_bfs_noalloc: needs %llu bytes of scratch, has %llu", (unsigned long long)o,
              (unsigned long long)kNoAllocScratchBytes);
    return GRE_NOBUFFER;
  }

  const uint32_t root = g->perm ? g->h_iperm[src] : src;
  RunTimer timer(g);
  GRE_CUDA(cudaMemcpyAsync(droot, &root, sizeof root, cudaMemcpyHostToDevice, g->stream));
  GRE_CUDA(cudaMemsetAsync(lv, 0xff, sizeof(int32_t) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(vis, 0, sizeof(uint32_t) * nwords, g->stream));
  GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), g->stream));
  k_bfs_seed<<<1, 32, 0, g->stream>>>(droot, 1, lv, vis, qa, g->off, c);
  BfsCounters h;
  GRE_CUDA(cudaMemcpyAsync(&h, c, sizeof h, cudaMemcpyDeviceToHost, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  uint64_t nf = h.next_count, mf = h.next_arcs;
  int64_t mu = (int64_t)g->m - (int64_t)mf;
  bool bottom_up = false;
  uint32_t *queue = qa, *nqueue = qb, *front = bits_a, *nbits = bits_b;
  int32_t d = 0;
  uint64_t scanned = 0;
  const int sms = num_sms();
  while (nf > 0) {
    if (!bottom_up && (double)mf > (double)mu / 15.0 && nf > 64) {
      GRE_CUDA(cudaMemsetAsync(front, 0, sizeof(uint32_t) * nwords, g->stream));
      k_queue_to_bits<<<grid_for(nf, 256), 256, 0, g->stream>>>(queue, nf, front);
      bottom_up = true;
    } else if (bottom_up && nf < n / 18) {
      GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), g->stream));
      k_bits_to_queue<<<grid_for(nwords, 256), 256, 0, g->stream>>>(n, front, queue, &c->next_count);
      bottom_up = false;
    }
    GRE_CUDA(cudaMemsetAsync(c, 0, sizeof(BfsCounters), g->stream));
    if (!bottom_up) {
      k_frontier_degrees<<<grid_for(nf, 256), 256, 0, g->stream>>>(queue, nf, g->off, deg);
      GRE_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, deg, prefix, nf + 1, g->stream));
      uint64_t total = 0;
      GRE_CUDA(cudaMemcpyAsync(&total, prefix + nf, sizeof total, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      if (total) {
        const int grid = (int)std::min<uint64_t>((total + 255) / 256, (uint64_t)sms * 16);
        k_td_expand<<<grid, 256, 0, g->stream>>>(queue, nf, prefix, total, g->off, g->col, vis, lv, d + 1, nqueue, c);
      }
      GRE_LAUNCH_CHECK();
      GRE_CUDA(cudaMemcpyAsync(&h, c, sizeof h, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      h.next_count = h.pad;
      scanned += total;
      std::swap(queue, nqueue);
    } else {
      k_bu_step<<<grid_for(nwords * 32, 256, 8), 256, 0, g->stream>>>(n, g->roff, g->rcol, g->off, front, nbits, vis, lv, d + 1, c);
      GRE_LAUNCH_CHECK();
      GRE_CUDA(cudaMemcpyAsync(&h, c, sizeof h, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      scanned += h.scanned;
      std::swap(front, nbits);
    }
    nf = h.next_count;
    mf = h.next_arcs;
    mu -= (int64_t)mf;
    ++d;
    stats_record(st, nf);
  }
  if (g->perm) {
    k_noalloc_unperm<<<grid_for(n, 256), 256, 0, g->stream>>>(n, g->iperm, lv, level);
    GRE_LAUNCH_CHECK();
  }
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = (uint32_t)(d > 0 ? d - 1 : 0);
    st->arcs_traversed = scanned;
  }
  return GRE_SUCCESS;
}

}  // extern "C"
