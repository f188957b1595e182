// Degree bins of a CSR/CSC and the autotuner that chooses their threads-per-row schedule.
//
// The schedule also decides whether the rows above cta_min are split at source windows (rows
// sorted by column only): their gathers then run window after window, so each window's share
// of the gathered array stays in L2 instead of being fetched again from HBM for every hub.
//
// The reference gives every active vertex to one worker thread and walks its arcs serially
// (Engine.hpp:592-625); on the GPU a row's arcs are spread over 1..32 lanes, a CTA, or several
// CTAs depending on its degree (rows.cuh).  Which degrees go to which width is a schedule
// (RowSchedule): arcs per lane for the narrow bins, the degree from which a row gets a whole CTA,
// and the chunk length of the longest rows.  The best schedule depends on the degree
// distribution, so it is measured: the first time a graph's bins are needed, each candidate
// schedule runs a PageRank-shaped pull superstep over that graph (an 8-byte gather per arc, the
// dominant access of the row kernels) and the fastest is kept.  The choice is cached per
// process under a key made from the degree distribution (arcs per power-of-two degree bucket,
// log2 n, log2 m), so graphs of the same shape - the batches of a run, replicas - tune once.
//
// GRE_TUNE=0 in the environment turns the measurement off (the default schedule is used), and
// graphs with fewer than 2^22 arcs always use the default: their supersteps are too short to
// time apart from launch overhead.  GRE_ROW_SCHEDULE=lane_arcs,cta_min,hub_chunk,seg_window
// imposes a schedule (tests use it to reach every kernel on small graphs).
#include <cub/cub.cuh>

#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "gre_internal.cuh"
#include "rows.cuh"

namespace gre {
namespace {

constexpr uint64_t kTuneMinArcs = 1ull << 22;
constexpr int kHistBuckets = 40;

__global__ void k_bin_of(uint64_t n, const uint64_t* __restrict__ off, uint8_t* __restrict__ bin, uint32_t lane_arcs,
                         uint64_t cta_min, uint64_t hub_chunk) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t d = off[v + 1] - off[v];
    uint8_t b = 255;
    if (d) {
      uint64_t lim = lane_arcs;
      for (int k = 0; k < 5; ++k, lim <<= 1) {
        if (d <= lim) {
          b = (uint8_t)k;
          break;
        }
      }
      if (b == 255) b = d <= cta_min ? 5 : d <= hub_chunk ? 6 : 7;
    }
    bin[v] = b;
  }
}

struct BinIs {
  const uint8_t* bin;
  uint8_t b;
  __host__ __device__ __forceinline__ bool operator()(const uint32_t& v) const { return bin[v] == b; }
};

__global__ void k_iota(uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    out[v] = (uint32_t)v;
}

// first and one-past-last arc of each listed row
__global__ void k_row_spans(uint64_t cnt, const uint32_t* __restrict__ rows, const uint64_t* __restrict__ off,
                            uint64_t* __restrict__ spans) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    spans[2 * i] = off[rows[i]];
    spans[2 * i + 1] = off[rows[i] + 1];
  }
}

// arcs per power-of-two degree bucket (bucket = bit length of the degree)
__global__ void k_degree_hist(uint64_t n, const uint64_t* __restrict__ off, unsigned long long* __restrict__ hist) {
  __shared__ unsigned long long h[kHistBuckets];
  for (int i = threadIdx.x; i < kHistBuckets; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t d = off[v + 1] - off[v];
    if (d) atomicAdd(&h[min(kHistBuckets - 1, 64 - __clzll((long long)d))], (unsigned long long)d);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kHistBuckets; i += blockDim.x)
    if (h[i]) atomicAdd(hist + i, h[i]);
}

struct ProbeGather {
  const uint32_t* __restrict__ col;
  const double* __restrict__ x;
  __device__ __forceinline__ double operator()(uint32_t, uint64_t a) const { return __ldg(x + __ldg(col + a)); }
};
struct ProbeStore {
  double* __restrict__ y;
  __device__ __forceinline__ void operator()(uint32_t v, double s) const { y[v] = s; }
};

int cub_temp(gre_graph g, size_t bytes, void** p) { return g->ws.get(WS_CUB, bytes, p); }

}  // namespace

void free_bins(DegreeBins& B) {
  cudaFree(B.rows);
  cudaFree(B.hub_chunk_row);
  cudaFree(B.hub_chunk_begin);
  cudaFree(B.hub_chunk_first);
  cudaFree(B.seg_rows);
  cudaFree(B.seg_first);
  cudaFree(B.seg_row);
  cudaFree(B.seg_begin);
  cudaFree(B.seg_end);
  cudaFree(B.seg_slot);
  B = DegreeBins();
}

namespace {

// first arc of each (row, window) whose column is >= window * seg (rows sorted by column);
// splits[r * (W + 1) + W] = end of row r
__global__ void k_window_splits(const uint32_t* __restrict__ rows, uint64_t nrows, const uint64_t* __restrict__ off,
                                const uint32_t* __restrict__ col, uint64_t seg, uint64_t W, uint64_t* __restrict__ splits) {
  const uint64_t total = nrows * (W + 1);
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = t / (W + 1), w = t - r * (W + 1);
    const uint32_t v = rows[r];
    uint64_t lo = off[v], hi = off[v + 1];
    if (w == W) {
      lo = hi;
    } else {
      const uint64_t key = w * seg;
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if ((uint64_t)col[mid] < key) lo = mid + 1;
        else hi = mid;
      }
    }
    splits[t] = lo;
  }
}

// Window-split chunks of the rows above cta_min (bins 6 and 7), see DegreeBins.
int build_segments(gre_graph g, DegreeBins& B, const uint64_t* off, const uint32_t* col) {
  const uint64_t seg = B.sched.seg_window;
  const uint64_t nrows = B.count[6] + B.count[7];
  if (!seg || !nrows) return GRE_SUCCESS;
  const uint64_t W = (g->n + seg - 1) / seg;
  const uint32_t* rows = B.rows + B.start[6];  // bins 6 and 7 are contiguous
  uint64_t* dsplits = nullptr;
  GRE_CUDA(cudaMalloc(&dsplits, sizeof(uint64_t) * nrows * (W + 1)));
  std::vector<uint64_t> sp(nrows * (W + 1));
  k_window_splits<<<grid_for(nrows * (W + 1), 256), 256, 0, g->stream>>>(rows, nrows, off, col, seg, W, dsplits);
  cudaError_t e = cudaMemcpyAsync(sp.data(), dsplits, sizeof(uint64_t) * sp.size(), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(dsplits);
  if (e != cudaSuccess) return cuda_status(e, "window splits", __FILE__, __LINE__);
  // the first arc of a row is its start: pieces of (row, window) of at most hub_chunk arcs; slots
  // row-major (a row's pieces in window order), processing order window-major
  const uint64_t piece = B.sched.hub_chunk;
  std::vector<uint64_t> first(nrows + 1, 0);
  for (uint64_t r = 0; r < nrows; ++r) {
    uint64_t k = 0;
    for (uint64_t w = 0; w < W; ++w) {
      const uint64_t a0 = sp[r * (W + 1) + w], a1 = sp[r * (W + 1) + w + 1];
      if (a1 > a0) k += (a1 - a0 + piece - 1) / piece;
    }
    first[r + 1] = first[r] + k;
  }
  const uint64_t nchunks = first[nrows];
  std::vector<uint32_t> crow(nchunks);
  std::vector<uint64_t> cbeg(nchunks), cend(nchunks), cslot(nchunks), next(first.begin(), first.end() - 1);
  std::vector<uint32_t> hrows(nrows);
  e = cudaMemcpy(hrows.data(), rows, sizeof(uint32_t) * nrows, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "window rows", __FILE__, __LINE__);
  uint64_t c = 0;
  for (uint64_t w = 0; w < W; ++w)
    for (uint64_t r = 0; r < nrows; ++r) {
      const uint64_t a0 = sp[r * (W + 1) + w], a1 = sp[r * (W + 1) + w + 1];
      for (uint64_t a = a0; a < a1; a += piece, ++c) {
        crow[c] = hrows[r];
        cbeg[c] = a;
        cend[c] = a + piece < a1 ? a + piece : a1;
        cslot[c] = next[r]++;
      }
    }
  B.seg_nrows = nrows;
  B.seg_nchunks = nchunks;
  e = cudaMalloc(&B.seg_rows, sizeof(uint32_t) * nrows);
  if (e == cudaSuccess) e = cudaMalloc(&B.seg_first, sizeof(uint64_t) * (nrows + 1));
  if (e == cudaSuccess) e = cudaMalloc(&B.seg_row, sizeof(uint32_t) * (nchunks ? nchunks : 1));
  if (e == cudaSuccess) e = cudaMalloc(&B.seg_begin, sizeof(uint64_t) * (nchunks ? nchunks : 1));
  if (e == cudaSuccess) e = cudaMalloc(&B.seg_end, sizeof(uint64_t) * (nchunks ? nchunks : 1));
  if (e == cudaSuccess) e = cudaMalloc(&B.seg_slot, sizeof(uint64_t) * (nchunks ? nchunks : 1));
  if (e == cudaSuccess) e = cudaMemcpy(B.seg_rows, hrows.data(), sizeof(uint32_t) * nrows, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B.seg_first, first.data(), sizeof(uint64_t) * (nrows + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nchunks) e = cudaMemcpy(B.seg_row, crow.data(), sizeof(uint32_t) * nchunks, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nchunks) e = cudaMemcpy(B.seg_begin, cbeg.data(), sizeof(uint64_t) * nchunks, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nchunks) e = cudaMemcpy(B.seg_end, cend.data(), sizeof(uint64_t) * nchunks, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nchunks) e = cudaMemcpy(B.seg_slot, cslot.data(), sizeof(uint64_t) * nchunks, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e, "window chunk upload", __FILE__, __LINE__);
  // partial slots the row kernels need (the hub-chunk arrays keep their own count)
  if (nchunks > B.n_partials) B.n_partials = nchunks;
  return GRE_SUCCESS;
}

}  // namespace

// Groups the rows of `off` by bin under `sched` (replacing what B held).
int build_bins(gre_graph g, DegreeBins& B, const uint64_t* off, const uint32_t* col, const RowSchedule& sched) {
  free_bins(B);
  B.sched = sched;
  const uint64_t n = g->n;
  uint8_t* bin = nullptr;
  uint32_t* iota = nullptr;
  uint64_t* nsel = nullptr;
  uint64_t* spans = nullptr;
  GRE_CUDA(cudaMalloc(&bin, n ? n : 1));
  cudaError_t e = cudaMalloc(&iota, sizeof(uint32_t) * (n ? n : 1));
  if (e == cudaSuccess) e = cudaMalloc(&nsel, sizeof(uint64_t) * DegreeBins::NB);
  if (e == cudaSuccess) e = cudaMalloc(&B.rows, sizeof(uint32_t) * (n ? n : 1));
  int st = e == cudaSuccess ? GRE_SUCCESS : cuda_status(e, "cudaMalloc (bins)", __FILE__, __LINE__);
  if (!st && n) {
    k_bin_of<<<grid_for(n, 256), 256, 0, g->stream>>>(n, off, bin, sched.lane_arcs, sched.cta_min, sched.hub_chunk);
    k_iota<<<grid_for(n, 256), 256, 0, g->stream>>>(n, iota);
    uint64_t base = 0;
    for (int b = 0; b < DegreeBins::NB && !st; ++b) {
      size_t tb = 0;
      BinIs pred{bin, (uint8_t)b};
      cub::DeviceSelect::If(nullptr, tb, iota, B.rows + base, nsel + b, n, pred, g->stream);
      void* tmp = nullptr;
      st = cub_temp(g, tb, &tmp);
      if (st) break;
      e = cub::DeviceSelect::If(tmp, tb, iota, B.rows + base, nsel + b, n, pred, g->stream);
      uint64_t cnt = 0;
      if (e == cudaSuccess) e = cudaMemcpyAsync(&cnt, nsel + b, sizeof cnt, cudaMemcpyDeviceToHost, g->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
      if (e != cudaSuccess) {
        st = cuda_status(e, "degree bins", __FILE__, __LINE__);
        break;
      }
      B.start[b] = base;
      B.count[b] = cnt;
      base += cnt;
    }
  }
  // chunks of the multi-CTA bin: only the spans of its rows come to the host
  if (!st && B.count[7]) {
    const uint64_t cnt = B.count[7];
    std::vector<uint64_t> hs(2 * cnt);
    e = cudaMalloc(&spans, sizeof(uint64_t) * 2 * cnt);
    if (e == cudaSuccess) {
      k_row_spans<<<grid_for(cnt, 256), 256, 0, g->stream>>>(cnt, B.rows + B.start[7], off, spans);
      e = cudaMemcpyAsync(hs.data(), spans, sizeof(uint64_t) * 2 * cnt, cudaMemcpyDeviceToHost, g->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) st = cuda_status(e, "hub chunks", __FILE__, __LINE__);
    if (!st) {
      std::vector<uint64_t> crow, cbeg, first;
      for (uint64_t i = 0; i < cnt; ++i) {
        first.push_back(crow.size());
        for (uint64_t a = hs[2 * i]; a < hs[2 * i + 1]; a += sched.hub_chunk) {
          crow.push_back(i);
          cbeg.push_back(a);
        }
      }
      first.push_back(crow.size());
      B.n_hub_chunks = crow.size();
      B.n_partials = crow.size();
      e = cudaMalloc(&B.hub_chunk_row, sizeof(uint64_t) * crow.size());
      if (e == cudaSuccess) e = cudaMalloc(&B.hub_chunk_begin, sizeof(uint64_t) * cbeg.size());
      if (e == cudaSuccess) e = cudaMalloc(&B.hub_chunk_first, sizeof(uint64_t) * first.size());
      if (e == cudaSuccess) e = cudaMemcpy(B.hub_chunk_row, crow.data(), sizeof(uint64_t) * crow.size(), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMemcpy(B.hub_chunk_begin, cbeg.data(), sizeof(uint64_t) * cbeg.size(), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMemcpy(B.hub_chunk_first, first.data(), sizeof(uint64_t) * first.size(), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) st = cuda_status(e, "hub chunk upload", __FILE__, __LINE__);
    }
  }
  cudaFree(bin);
  cudaFree(iota);
  cudaFree(nsel);
  cudaFree(spans);
  if (!st) st = build_segments(g, B, off, col);
  if (st) {
    free_bins(B);
    return st;
  }
  B.ready = true;
  return GRE_SUCCESS;
}

namespace {

int degree_key(gre_graph g, const uint64_t* off, std::string* key) {
  unsigned long long* dh = nullptr;
  GRE_CUDA(cudaMalloc(&dh, sizeof(unsigned long long) * kHistBuckets));
  cudaError_t e = cudaMemsetAsync(dh, 0, sizeof(unsigned long long) * kHistBuckets, g->stream);
  unsigned long long h[kHistBuckets] = {};
  if (e == cudaSuccess) {
    k_degree_hist<<<grid_for(g->n, 256), 256, 0, g->stream>>>(g->n, off, dh);
    e = cudaMemcpyAsync(h, dh, sizeof h, cudaMemcpyDeviceToHost, g->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(dh);
  if (e != cudaSuccess) return cuda_status(e, "degree histogram", __FILE__, __LINE__);
  auto lg = [](uint64_t x) { int b = 0; while (x > 1) { x >>= 1; ++b; } return b; };
  char buf[32];
  snprintf(buf, sizeof buf, "n%d m%d:", lg(g->n), lg(g->m));
  *key = buf;
  for (int i = 0; i < kHistBuckets; ++i) {  // share of arcs per bucket, in percent
    snprintf(buf, sizeof buf, "%d,", (int)((200.0 * (double)h[i] / (double)(g->m ? g->m : 1) + 1.0) / 2.0));
    *key += buf;
  }
  return GRE_SUCCESS;
}

// Times five probe supersteps under the current bins; returns the fastest of the last four, in ms
// (candidates 1-2% apart flipped with the fastest of two).
int probe(gre_graph g, const DegreeBins& B, const uint64_t* off, const uint32_t* col, const double* x, double* y, float* best_ms) {
  double* partial = nullptr;
  GRE_CUDA(cudaMalloc(&partial, sizeof(double) * (B.n_partials + 1)));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int st = e == cudaSuccess ? GRE_SUCCESS : cuda_status(e, "probe events", __FILE__, __LINE__);
  float best = 1e30f;
  for (int r = 0; r < 5 && !st; ++r) {
    cudaEventRecord(e0, g->stream);
    st = rows::reduce_rows(B, off, ProbeGather{col, x}, ProbeStore{y}, partial, g->stream);
    cudaEventRecord(e1, g->stream);
    e = cudaEventSynchronize(e1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess && !st) st = cuda_status(e, "probe", __FILE__, __LINE__);
    if (r > 0 && ms < best) best = ms;  // the first run warms the caches
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(partial);
  *best_ms = best;
  return st;
}

int tune(gre_graph g, DegreeBins& B, const uint64_t* off, const uint32_t* col, bool sorted, RowSchedule* best) {
  double *x = nullptr, *y = nullptr;
  GRE_CUDA(cudaMalloc(&x, sizeof(double) * g->n));
  cudaError_t e = cudaMalloc(&y, sizeof(double) * g->n);
  if (e == cudaSuccess) e = cudaMemsetAsync(x, 0, sizeof(double) * g->n, g->stream);
  int st = e == cudaSuccess ? GRE_SUCCESS : cuda_status(e, "tuner buffers", __FILE__, __LINE__);
  float best_ms = 1e30f;
  // RMAT-26, PageRank superstep with a fixed schedule (lane_arcs / cta_min / hub_chunk): 4 / 16384 /
  // 65536 8.93 ms, 8 / 8192 8.94, 8 / 16384 8.82, 32 / 16384 8.81, 16 / 16384 8.69, 8 / 65536 8.70,
  // 16 / 65536 / 131072 8.63
  for (uint32_t lane_arcs : {2u, 4u, 8u, 16u}) {
    for (uint64_t cta_min : {4096ull, 16384ull, 65536ull}) {
      if (st) break;
      RowSchedule cand;
      cand.lane_arcs = lane_arcs;
      cand.cta_min = cta_min;
      cand.hub_chunk = cta_min > 32768 ? 2 * cta_min : 65536;
      float ms = 0;
      st = build_bins(g, B, off, col, cand);
      if (!st) st = probe(g, B, off, col, x, y, &ms);
      if (!st && ms < best_ms) {
        best_ms = ms;
        *best = cand;
      }
    }
  }
  // source windows for the rows above cta_min, when the rows are sorted and the gathered
  // values (8 bytes per vertex) outgrow a window of 64 MB (half the L2).  On RMAT-26 the windows
  // measured no faster (the hub rows' gathers are bound by L2 request rate, not by misses), so
  // one window size is tried, to keep the tuning short.
  for (uint64_t window : {1ull << 23}) {
    if (st || !sorted || g->n <= window) break;
    RowSchedule cand = *best;
    cand.seg_window = window;
    float ms = 0;
    st = build_bins(g, B, off, col, cand);
    if (!st) st = probe(g, B, off, col, x, y, &ms);
    if (!st && ms < best_ms) {
      best_ms = ms;
      *best = cand;
    }
  }
  cudaFree(x);
  cudaFree(y);
  return st;
}

std::mutex g_tuned_mu;
std::map<std::string, RowSchedule> g_tuned;

bool tuning_enabled() {
  const char* e = getenv("GRE_TUNE");
  return !(e && e[0] == '0');
}

}  // namespace

int ensure_bins(gre_graph g, bool in) {
  DegreeBins& B = in ? g->bins_in : g->bins_out;
  if (B.ready) return GRE_SUCCESS;
  const uint64_t* off = in ? g->roff : g->off;
  const uint32_t* col = in ? g->rcol : g->col;
  const bool sorted = in && !g->symmetric() ? true : g->csr_sorted;  // the CSC is built sorted
  RowSchedule sched;  // default
  if (const char* e = getenv("GRE_ROW_SCHEDULE")) {  // "lane_arcs,cta_min,hub_chunk,seg_window": a fixed schedule
    unsigned long long a = 0, c = 0, h = 0, w = 0;
    if (sscanf(e, "%llu,%llu,%llu,%llu", &a, &c, &h, &w) != 4 || a < 1 || a > 64 || c < 16 * a || h < c || h == 0) {
      set_error("GRE_ROW_SCHEDULE must be lane_arcs,cta_min,hub_chunk,seg_window with 16*lane_arcs <= cta_min <= hub_chunk");
      return GRE_INVALID_ARG;
    }
    sched.lane_arcs = (uint32_t)a;
    sched.cta_min = c;
    sched.hub_chunk = h;
    sched.seg_window = sorted ? w : 0;
    return build_bins(g, B, off, col, sched);
  }
  if (tuning_enabled() && g->m >= kTuneMinArcs) {
    std::string key;
    GRE_CHECK(degree_key(g, off, &key));
    key += sorted ? "sorted" : "unsorted";
    bool found = false;
    {
      std::lock_guard<std::mutex> lock(g_tuned_mu);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) {
        sched = it->second;
        found = true;
      }
    }
    if (!found) {
      GRE_CHECK(tune(g, B, off, col, sorted, &sched));
      std::lock_guard<std::mutex> lock(g_tuned_mu);
      g_tuned[key] = sched;
    }
    if (B.ready && B.sched.lane_arcs == sched.lane_arcs && B.sched.cta_min == sched.cta_min &&
        B.sched.hub_chunk == sched.hub_chunk && B.sched.seg_window == sched.seg_window)
      return GRE_SUCCESS;  // the last candidate tried is the one kept
  }
  return build_bins(g, B, off, col, sched);
}

}  // namespace gre

extern "C" int gre_row_schedule(gre_graph g, int in, uint32_t* lane_arcs, uint64_t* cta_min, uint64_t* hub_chunk,
                                uint64_t* seg_window) {
  using namespace gre;
  if (!g || !lane_arcs || !cta_min || !hub_chunk || !seg_window) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  GRE_CHECK(ensure_bins(g, in != 0));
  const DegreeBins& B = in ? g->bins_in : g->bins_out;
  *lane_arcs = B.sched.lane_arcs;
  *cta_min = B.sched.cta_min;
  *hub_chunk = B.sched.hub_chunk;
  *seg_window = B.seg_nchunks ? B.sched.seg_window : 0;
  return GRE_SUCCESS;
}
