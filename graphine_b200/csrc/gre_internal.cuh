// Internal definitions of libgre_gpu.so: the graph handle, per-graph scratch workspace, error
// plumbing and small device helpers shared by the kernel translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "../../include/gre_gpu.h"

namespace gre {

// ---------------------------------------------------------------------------------------------
// Errors: every ABI call returns a status; the text of the last failure is kept per thread.
// ---------------------------------------------------------------------------------------------
void set_error(const char* fmt, ...);
void clear_error();
int cuda_status(cudaError_t e, const char* what, const char* file, int line);

#define GRE_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t gre_e_ = (call);                                                \
    if (gre_e_ != cudaSuccess) return ::gre::cuda_status(gre_e_, #call, __FILE__, __LINE__); \
  } while (0)

#define GRE_CHECK(expr)        \
  do {                         \
    int gre_s_ = (expr);       \
    if (gre_s_) return gre_s_; \
  } while (0)

#define GRE_LAUNCH_CHECK() GRE_CUDA(cudaGetLastError())

// ---------------------------------------------------------------------------------------------
// Scratch workspace: named device buffers owned by a graph handle, grown on demand and kept
// until the handle is freed, so repeated runs do no allocation.
// ---------------------------------------------------------------------------------------------
enum WsSlot {
  WS_A = 0, WS_B, WS_C, WS_D, WS_E, WS_F, WS_G, WS_H, WS_I, WS_J, WS_K, WS_L, WS_M, WS_N,
  WS_COUNTERS,   // small per-run counters (device-side)
  WS_CUB,        // CUB temporary storage
  WS_OUTBUF,     // device staging of results bound for host memory
  WS_OUTBUF2,
  // betweenness state (kept apart from the slots the BFS routines use)
  WS_BC0, WS_BC1, WS_BC2, WS_BC3, WS_BC4, WS_BC5, WS_BC6, WS_BC7,
  WS_PERM_OUT,   // results in internal order, before un-permuting (relabelled graphs)
  WS_PERM_IN,    // inputs permuted to internal order
  WS_PERM_IN2,
  WS_PERM_OFF,   // caller-order row offsets
  WS_SSSP_L,     // SSSP: vertices with light arcs (bitmap)
  WS_SSSP_H,     // SSSP: vertices with heavy arcs (bitmap)
  WS_NSLOTS
};

struct Workspace {
  void* ptr[WS_NSLOTS] = {};
  size_t bytes[WS_NSLOTS] = {};
  int get(int slot, size_t nbytes, void** out);
  void release();
};

// Degree bins of one adjacency (rows grouped by the number of lanes that process them).
// Threads-per-row schedule of the degree bins: bin b < 5 (2^b lanes per row) takes rows of up to
// lane_arcs * 2^b arcs, bin 5 (a warp) rows up to cta_min arcs, bin 6 (a CTA) rows up to
// hub_chunk arcs, bin 7 the longer rows in chunks of hub_chunk arcs.  Chosen per graph by the
// autotuner (bins.cu) from the degree distribution.
struct RowSchedule {
  uint32_t lane_arcs = 4;
  uint64_t cta_min = 4096;
  uint64_t hub_chunk = 65536;
  // Rows above cta_min split at source windows of seg_window vertices (0: not split); needs
  // rows sorted by column.  Their chunks run window after window, so the values gathered by
  // all of them come from one window at a time, which stays in L2.
  uint64_t seg_window = 0;
};

struct DegreeBins {
  bool ready = false;
  RowSchedule sched;
  static const int NB = 8;  // 1,2,4,8,16,32 lanes, CTA per row, multi-CTA per row
  uint64_t count[NB] = {};
  uint64_t start[NB] = {};   // offsets into `rows`
  uint32_t* rows = nullptr;  // row ids grouped by bin (device)
  uint64_t n_hub_chunks = 0; // chunks of the multi-CTA bin (entries of hub_chunk_row / _begin)
  uint64_t n_partials = 0;   // partial-sum slots the row kernels need: the hub chunks, or the
                             // window chunks when the schedule splits rows by source window
  uint64_t* hub_chunk_row = nullptr;   // per chunk: index into the multi-CTA bin
  uint64_t* hub_chunk_begin = nullptr; // per chunk: first arc
  uint64_t* hub_chunk_first = nullptr; // per multi-CTA row: first chunk id (size count+1)
  // Window-split rows (sched.seg_window != 0): the rows above cta_min (bins 6 and 7).  Chunk c,
  // in processing order (window-major), covers arcs [seg_begin[c], seg_end[c]) of vertex
  // seg_row[c] and writes its partial sum to slot seg_slot[c]; row i of seg_rows adds slots
  // seg_first[i] .. seg_first[i+1]-1 in order (its chunks in window order).
  uint64_t seg_nrows = 0, seg_nchunks = 0;
  uint32_t* seg_rows = nullptr;
  uint64_t* seg_first = nullptr;
  uint32_t* seg_row = nullptr;
  uint64_t* seg_begin = nullptr;
  uint64_t* seg_end = nullptr;
  uint64_t* seg_slot = nullptr;
};

// Rows longer than `ch` arcs split into fixed chunks of `ch` arcs from the row start.  Partial
// sums of the chunks are added in chunk order, which fixes the association order of a row's
// sum independently of how many threads work on it.
struct ChunkTable {
  bool ready = false;
  uint64_t ch = 0;
  uint64_t nrows = 0, nchunks = 0;
  uint32_t* rows = nullptr;         // long rows
  uint64_t* chunk_row = nullptr;    // chunk -> index into rows
  uint64_t* chunk_begin = nullptr;  // chunk -> first arc
  uint64_t* first = nullptr;        // long row i -> first chunk (nrows + 1 entries)
};

}  // namespace gre

struct gre_graph_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint64_t n = 0, m = 0;
  uint32_t flags = 0;  // gre_dir | gre_graph_flags
  // CSR (out-arcs)
  uint64_t* off = nullptr;
  uint32_t* col = nullptr;
  // CSC (in-arcs); alias the CSR when the graph is symmetric
  uint64_t* roff = nullptr;
  uint32_t* rcol = nullptr;
  uint64_t* rarc = nullptr;  // CSC slot -> CSR arc id (built on demand)
  uint32_t* outdeg = nullptr;
  uint32_t* indeg = nullptr;  // aliases outdeg when symmetric
  bool csr_sorted = false;    // every CSR row lists its columns in increasing order (the CSC always does)
  // weights
  uint32_t* w32 = nullptr;
  double w32_mean = -1.0;  // mean of w32, computed on first use (-1: unknown)
  // the weight of every arc u->v equals that of v->u (a symmetric graph with weights of the
  // undirected edge, as gre_graph_set_weights_hash makes them); lets SSSP pull over a vertex's
  // own arcs instead of pushing along its neighbours'
  bool w32_symmetric = false;
  // SSSP light/heavy arc split for bucket width `delta` (sssp.cu): each row's arcs reordered so
  // the light ones (w < delta) come first; heavy ones start at lsplit[v].  Built on first use,
  // dropped when the weights or the arc order change.
  struct SsspSplit {
    uint32_t* col = nullptr;
    uint32_t* w = nullptr;
    uint64_t* lsplit = nullptr;
    uint32_t delta = 0;
    void release() {
      cudaFree(col);
      cudaFree(w);
      cudaFree(lsplit);
      *this = SsspSplit();
    }
  } sssp_split;
  double* w64 = nullptr;
  double* rw64 = nullptr;  // FP64 weights in CSC order (built on demand)
  uint64_t max_outdeg = 0, max_indeg = 0;
  gre::Workspace ws;
  gre::DegreeBins bins_in, bins_out;
  // SSSP's binned passes, when the tuned schedule gives rows more than 8 arcs per lane or a warp
  // above 16384 arcs (sssp_bins): the pushes are latency-bound and want short chains per lane
  gre::DegreeBins bins_sssp;
  // Degree-ordered relabelling (GRE_GRAPH_REORDER / gre_graph_reorder): every internal array
  // uses internal ids; perm[i] is the caller's id of internal vertex i (the reference's
  // lvid2vid, DistributedGraph.hpp:57-59) and iperm its inverse.  Null when not relabelled.
  uint32_t* perm = nullptr;
  uint32_t* iperm = nullptr;
  std::vector<uint32_t> h_iperm;  // host copy, to map source ids
  // Relabelled rows are sorted by internal neighbour id; arc_rank[a] is the position of internal
  // arc a within its caller row (caller arc = caller_off[perm[row]] + arc_rank[a]).
  uint32_t* arc_rank = nullptr;
  gre::ChunkTable bc_chunks;       // in-arc rows longer than 512 arcs (betweenness)
  uint64_t* bc_fpool = nullptr;    // per-level frontier words of the batched betweenness
  uint64_t bc_fpool_levels = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_caller = nullptr;  // orders the stream after the caller's legacy-stream work (use_graph)
  bool symmetric() const { return (flags & GRE_GRAPH_SYMMETRIC) != 0; }
};

namespace gre {

// ---------------------------------------------------------------------------------------------
// Host helpers
// ---------------------------------------------------------------------------------------------
inline int grid_for(uint64_t work, int block, int max_blocks_per_sm = 8) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  uint64_t b = (work + block - 1) / block;
  uint64_t cap = (uint64_t)sms * max_blocks_per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

int num_sms();

// Pointer on the device?  (cudaPointerGetAttributes: device or managed memory)
bool is_device_ptr(const void* p);

// Make the graph's device current.
int use_graph(gre_graph g);

// Input array of `count` T: device pointer returned as is, host data staged into `slot`.
template <class T>
int stage_input(gre_graph g, const T* p, uint64_t count, int slot, const T** dev) {
  if (!p) {
    *dev = nullptr;
    return GRE_SUCCESS;
  }
  if (is_device_ptr(p)) {
    *dev = p;
    return GRE_SUCCESS;
  }
  void* d = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &d));
  if (count) GRE_CUDA(cudaMemcpyAsync(d, p, sizeof(T) * count, cudaMemcpyHostToDevice, g->stream));
  *dev = (const T*)d;
  return GRE_SUCCESS;
}

// Output array: a device pointer is written in place; a host pointer gets a device staging
// buffer in `slot` and is filled by finish_output.
template <class T>
int prepare_output(gre_graph g, T* p, uint64_t count, int slot, T** dev) {
  if (is_device_ptr(p)) {
    *dev = p;
    return GRE_SUCCESS;
  }
  void* d = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &d));
  *dev = (T*)d;
  return GRE_SUCCESS;
}

template <class T>
int finish_output(gre_graph g, T* p, const T* dev, uint64_t count) {
  if ((const void*)p != (const void*)dev && count)
    GRE_CUDA(cudaMemcpyAsync(p, dev, sizeof(T) * count, cudaMemcpyDeviceToHost, g->stream));
  return GRE_SUCCESS;
}

// Timing of one ABI call on the graph's stream.
struct RunTimer {
  gre_graph g;
  explicit RunTimer(gre_graph gg) : g(gg) { cudaEventRecord(g->ev0, g->stream); }
  int stop(gre_stats* st) {
    GRE_CUDA(cudaEventRecord(g->ev1, g->stream));
    GRE_CUDA(cudaEventSynchronize(g->ev1));
    float ms = 0;
    GRE_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    if (st) st->device_ms = ms;
    return GRE_SUCCESS;
  }
};

// Graph construction steps (graph.cu): an empty handle on `device`; degrees, maxima and CSC once
// off/col are on the device; degree-ordered relabelling with sorted rows; teardown.
int new_graph(int device, uint32_t flags, gre_graph* out);
int finish_graph(gre_graph g);
int reorder_graph(gre_graph g);
void destroy_graph(gre_graph g);
// Frees a half-built handle on an error path unless released.
struct GraphGuard {
  gre_graph g;
  ~GraphGuard() {
    if (g) destroy_graph(g);
  }
  gre_graph release() {
    gre_graph r = g;
    g = nullptr;
    return r;
  }
};
// <prefix>.meta + <prefix>.edges.<i> parsed on the device (ingest.cu).
int device_ingest(const char* prefix, uint32_t flags, int device, gre_graph* out);
int device_ingest_parts(const char* prefix, uint32_t nparts, uint32_t flags, int device, gre_graph* out);

void launch_count_add(long long k);

// A fixed sequence of launches on one stream, recorded once into a CUDA graph and replayed:
// one host call per replay instead of one per kernel (supersteps whose shape does not depend
// on data, e.g. a period of PageRank iterations).  The body may only enqueue work on the
// stream (kernels, memsets, device-to-device copies): no allocation, no host synchronisation.
class Recorded {
 public:
  Recorded() = default;
  Recorded(const Recorded&) = delete;
  Recorded& operator=(const Recorded&) = delete;
  ~Recorded() {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
  }
  template <class F>
  int record(cudaStream_t s, F&& body) {
    const unsigned long long before = gre_launch_count();
    GRE_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int st = body();
    const cudaError_t e = cudaStreamEndCapture(s, &graph_);
    kernels_ = (long long)(gre_launch_count() - before);
    launch_count_add(-kernels_);
    if (st) return st;
    GRE_CUDA(e);
    GRE_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
    return GRE_SUCCESS;
  }
  int replay(cudaStream_t s) {
    GRE_CUDA(cudaGraphLaunch(exec_, s));
    launch_count_add(kernels_);
    return GRE_SUCCESS;
  }

 private:
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  long long kernels_ = 0;
};

inline void stats_reset(gre_stats* st) {
  if (!st) return;
  st->supersteps = 0;
  st->n_recorded = 0;
  st->arcs_traversed = 0;
  st->traversed_edges = 0;
  st->algo_bytes = 0;
  st->device_ms = 0;
  st->plugin_value = 0;
  st->plugin_count = 0;
}
inline void stats_record(gre_stats* st, uint64_t active) {
  if (st && st->n_recorded < GRE_MAX_RECORDED_SUPERSTEPS) st->active[st->n_recorded++] = active;
}

// Degree bins of the CSC (in = true) or CSR; built once per graph.
int ensure_bins(gre_graph g, bool in);
// Degree bins of the rows of `off` (g->n rows) under a fixed schedule (replacing what B held).
int build_bins(gre_graph g, DegreeBins& B, const uint64_t* off, const uint32_t* col, const RowSchedule& sched);
void free_bins(DegreeBins& B);
// CSC slot -> CSR arc map; built once per graph.
int ensure_rarc(gre_graph g);
// Undirected edge count with both endpoints in a reached set (Graph500 TEPS numerator).
int count_reached_edges(gre_graph g, const int32_t* level, uint64_t* edges, uint64_t rows = 1);
// SSSP bucket width: 3/8 of the mean uint32 weight (GRE_SSSP_DELTA overrides; 0 = no buckets).
int sssp_delta(gre_graph g, uint32_t* delta);
// Heads a partitioned relaxation owns itself (sssp.cu offer forms): heads in [lo, lo + len) are
// relaxed in place, as in the one-GPU pass (dist[head - lo] lowered by atomic min, the head's bit
// set in `pend` when it has out-arcs); only the other heads are offered.  len = 0: none.
struct OwnHeads {
  uint64_t lo = 0, len = 0;
  uint32_t* dist = nullptr;
  uint32_t* pend = nullptr;
  const uint32_t* outdeg = nullptr;
};
// One edge-balanced relaxation pass (sssp.cu): the frontier `queue` (nq vertices, exclusive
// scan `prefix` of their arc counts, `total` arcs starting at base[u]) offers srcdist[u] + w to
// dist[head] (atomic min), and sets the head's bit in `changed` (may be null) on improvement.
// srcdist == dist: the one-GPU relaxation; otherwise dist is a separate offer array, an offer at
// or above known[head] (an upper bound of the head's distance; may be null) is dropped, and the
// heads in `own` are relaxed in place.  tstart holds ceil(total / sssp_tile_arcs()) entries;
// error is set if a tile holds too many owners.
uint64_t sssp_tile_arcs();
// The binned form of a relaxation pass as offers (sssp.cu): every row of the bins whose bit is set
// in `front` offers srcdist[row] + w over its light arcs [off[row], lend[row]) (heavy: [lend[row],
// off[row+1])) into `offers` (atomic min), setting the entry's bit in `touched` (may be null);
// offers at or above known[head] (may be null) are dropped, the heads in `own` are relaxed in
// place; `arcs` (may be null) counts the arcs.
int sssp_relax_binned_offer(cudaStream_t stream, const DegreeBins& B, const uint32_t* front, const uint64_t* off,
                            const uint64_t* lend, bool heavy, const uint32_t* col, const uint32_t* w, const uint32_t* srcdist,
                            uint32_t* offers, uint32_t* touched, const uint32_t* known, const OwnHeads& own,
                            unsigned long long* arcs);
// The pull form of a pass (sssp.cu; symmetric graph with symmetric weights): every row whose
// dist[row] >= lo takes the smallest srcdist[u] + w over its light (heavy) arcs to columns u set
// in `front`; an improvement lowers dist[row] and sets the row's bit in `changed`.  counts[0] +=
// arcs scanned, counts[1] += frontier hits.
int sssp_pull_binned(cudaStream_t stream, const DegreeBins& B, const uint32_t* front, const uint64_t* off, const uint64_t* lend,
                     bool heavy, const uint32_t* col, const uint32_t* w, const uint32_t* srcdist, uint32_t* dist, uint32_t* changed,
                     uint32_t lo, unsigned long long* counts);
// Light/heavy split of `rows` rows for bucket width delta (sssp.cu): light arcs (w < delta) first.
int sssp_split_rows(cudaStream_t stream, uint64_t rows, const uint64_t* off, const uint32_t* col, const uint32_t* w, uint32_t delta,
                    uint32_t* ocol, uint32_t* ow, uint64_t* lend);
// Frontiers of at least n / sssp_binned_divisor() vertices go through the degree bins (0: never);
// whether heavy passes may pull (GRE_SSSP_BINNED, GRE_SSSP_PULL).
// The bins SSSP's binned passes use (sssp.cu): the graph's CSR (in = false) or CSC bins, or a copy
// with at most 8 arcs per lane and a CTA from 16384 arcs when the tuned schedule is wider.
int sssp_bins(gre_graph g, bool in, const DegreeBins** out);
uint64_t sssp_binned_divisor();
bool sssp_pull_enabled();
// A heavy pass with at least m / sssp_pull_arcs_divisor() arcs pulls whatever its member count
// (GRE_SSSP_PULL_ARCS; 0: never by arcs).
uint64_t sssp_pull_arcs_divisor();
int sssp_relax_tiles(cudaStream_t stream, const uint32_t* queue, uint64_t nq, const uint64_t* prefix, uint64_t total,
                     uint32_t* tstart, const uint64_t* base, const uint32_t* col, const uint32_t* w, const uint32_t* srcdist,
                     uint32_t* dist, uint32_t* changed, uint32_t* error, const uint32_t* known, const OwnHeads& own);
// Direction-optimising BFS levels from device roots (uses slots WS_A..WS_G, WS_COUNTERS, WS_CUB).
int bfs_levels(gre_graph g, const uint32_t* droots, uint32_t nroots, int32_t* level, gre_stats* st, bool record);

// ---------------------------------------------------------------------------------------------
// Relabelled graphs: caller ids <-> internal ids.  All no-ops when g->perm is null.
// ---------------------------------------------------------------------------------------------
// Caller vertex ids (host) -> internal ids, validated against n.
int map_ids(gre_graph g, std::vector<uint32_t>* ids, const char* what);
// Output of `rows` x n values: returns in *internal the buffer the kernels should write (the
// output itself when not relabelled) and later un-permutes it into `out`.
int perm_out_begin(gre_graph g, void* out_dev, uint64_t rows, size_t elem, void** internal);
int perm_out_end(gre_graph g, const void* internal, void* out_dev, uint64_t rows, size_t elem);
// Input of n values in caller order -> internal order (returns the input when not relabelled).
int perm_in(gre_graph g, const void* in_dev, size_t elem, int slot, const void** internal);
// Per-arc arrays: caller CSR order <-> internal arc order.
int arcs_to_internal(gre_graph g, const void* in_dev, void* out_dev, size_t elem);
int arcs_to_caller(gre_graph g, const void* in_dev, void* out_dev, size_t elem);
// The CSR in caller ids and caller row order (arc order within a row as stored).
int caller_csr(gre_graph g, uint64_t* off_out, uint32_t* col_out);

// ---------------------------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

template <class T>
__device__ __forceinline__ T ldg_nc(const T* p) { return __ldg(p); }

// Warp-aggregated append of one item per active lane into a queue.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
  const uint32_t mask = __ballot_sync(0xffffffffu, want);
  if (!mask) return 0xffffffffu;
  const uint32_t lane = lane_id();
  const uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  return want ? base + __popc(mask & ((1u << lane) - 1u)) : 0xffffffffu;
}

// Per-warp staging of appends to K global lists.  A pass that appends most of the graph through
// warp_append makes one global atomic per 32 items on the same few counters, and those atomics
// bound it; here each warp gathers its items in shared memory (CAP per list) and moves them out
// with one atomic per CAP items and coalesced stores.  Every call is warp-uniform (all 32 lanes,
// the same k); `buf` is this warp's K * CAP words of shared memory.  The order of items in a
// list is not kept (callers treat lists as sets).
template <int K, int CAP>
struct WarpLists {
  uint32_t* buf;
  uint32_t held[K];
  __device__ __forceinline__ explicit WarpLists(uint32_t* b) : buf(b) {
#pragma unroll
    for (int k = 0; k < K; ++k) held[k] = 0;
  }
  template <int k>
  __device__ __forceinline__ void push(bool want, uint32_t v, uint32_t* counter, uint32_t* list) {
    const uint32_t mask = __ballot_sync(0xffffffffu, want);
    if (!mask) return;
    if (held[k] + 32 > CAP) flush<k>(counter, list);
    if (want) buf[k * CAP + held[k] + __popc(mask & ((1u << lane_id()) - 1u))] = v;
    held[k] += __popc(mask);
  }
  template <int k>
  __device__ __forceinline__ void flush(uint32_t* counter, uint32_t* list) {
    __syncwarp();
    const uint32_t c = held[k];
    if (!c) return;
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(counter, c);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t i = lane_id(); i < c; i += 32) list[base + i] = buf[k * CAP + i];
    __syncwarp();
    held[k] = 0;
  }
};
#endif

}  // namespace gre
