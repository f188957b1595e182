// Device-side ingress of <prefix>.meta + <prefix>.edges.<i> (GraphIngress::loadMetaFromFile /
// loadEdgesFromFiles, GraphIngress.hpp:323-328, 511-723; CSR build LocalGraph.hpp:66-107).
//
// The reference parses the text on the host (strtoul per token) and builds the CSR with
// per-thread scans of the whole edge list; at RMAT-26 that is ~36 GB of text.  Here the host
// only reads bytes: each file streams through two pinned buffers in chunks of whole lines, the
// next chunk is read while the GPU parses the current one, and on the GPU
//   1. line starts are selected (position 0 and every byte after a '\n'),
//   2. one thread per line parses "u v" with the reference loader's rules (blank lines and
//      lines starting with '#' skipped, a trailing '\r' ignored, anything else malformed),
//   3. the valid (u, v) pairs are compacted in file order and appended to the edge list,
// and at the end one stable radix sort by source gives the CSR with file order kept within a
// source - the order GraphInCSR::build produces.
//
// Errors keep the loader's codes: a malformed line is GRE_IO_ERROR, an id above 2^32-1 or not
// below n (from .meta) is GRE_INVALID_ARG; the first bad line in file order decides.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "gre_internal.cuh"

namespace gre {
namespace {

constexpr uint64_t kSkip = ~0ull;  // parse output of a skipped or bad line

struct LineStart {
  const char* buf;
  __device__ __forceinline__ bool operator()(const uint32_t& i) const { return i == 0 || buf[i - 1] == '\n'; }
};
struct NotSkip {
  __device__ __forceinline__ bool operator()(const uint64_t& x) const { return x != kSkip; }
};

// Line i spans [starts[i], end) where end is the '\n' that closes it (the chunk ends with one).
__global__ void k_parse_lines(const char* __restrict__ buf, uint64_t len, const uint32_t* __restrict__ starts, uint64_t nlines,
                              uint64_t line0, uint64_t nv, uint64_t* __restrict__ out, unsigned long long* __restrict__ first_err) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlines; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = starts[i];
    uint64_t lend = (i + 1 < nlines ? (uint64_t)starts[i + 1] : len) - 1;  // the '\n'
    if (lend > b && buf[lend - 1] == '\r') --lend;
    uint64_t result = kSkip;
    int err = 0;
    if (lend != b && buf[b] != '#') {
      uint64_t q = b, vals[2] = {0, 0};
      for (int k = 0; k < 2 && !err; ++k) {
        while (q < lend && (buf[q] == ' ' || buf[q] == '\t')) ++q;
        if (q >= lend || buf[q] < '0' || buf[q] > '9') {
          err = GRE_IO_ERROR;
          break;
        }
        uint64_t x = 0;
        while (q < lend && buf[q] >= '0' && buf[q] <= '9') {
          x = x * 10 + (uint64_t)(buf[q] - '0');
          if (x > 0xffffffffull) {
            err = GRE_INVALID_ARG;
            break;
          }
          ++q;
        }
        vals[k] = x;
      }
      if (!err) {
        while (q < lend && (buf[q] == ' ' || buf[q] == '\t')) ++q;
        if (q != lend) err = GRE_IO_ERROR;  // a third token (e.g. a weight) is not this format
        else if (vals[0] >= nv || vals[1] >= nv) err = GRE_INVALID_ARG;
        else result = (vals[0] << 32) | vals[1];
      }
    }
    out[i] = result;
    if (err) atomicMin(first_err, (unsigned long long)(((line0 + i) << 4) | (uint64_t)err));
  }
}

__global__ void k_split_packed(uint64_t m, const uint64_t* __restrict__ keys, uint32_t* __restrict__ col) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
    col[i] = (uint32_t)keys[i];
}

// off[v] = first position whose source (high word) is >= v
__global__ void k_offsets_by_high(uint64_t n, uint64_t m, const uint64_t* __restrict__ keys, uint64_t* __restrict__ off) {
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

uint64_t chunk_bytes() {
  const char* e = getenv("GRE_INGEST_CHUNK");  // smaller chunks exercise the line carry-over
  uint64_t c = e ? strtoull(e, nullptr, 10) : (64ull << 20);
  return std::max<uint64_t>(c, 64);
}

// Everything the streaming parse holds; freed on every exit path.
struct Ingest {
  char* pin[2] = {nullptr, nullptr};
  char* dbuf = nullptr;
  uint32_t* starts = nullptr;
  uint64_t* parsed = nullptr;
  uint64_t* edges = nullptr;
  uint64_t cap = 0, m = 0;
  unsigned long long* counters = nullptr;  // [0] lines selected, [1] edges selected, [2] first error
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  ~Ingest() {
    cudaFreeHost(pin[0]);
    cudaFreeHost(pin[1]);
    cudaFree(dbuf);
    cudaFree(starts);
    cudaFree(parsed);
    cudaFree(edges);
    cudaFree(counters);
    cudaFree(tmp);
  }
  int scratch(size_t bytes) {
    if (bytes <= tmp_bytes) return GRE_SUCCESS;
    cudaFree(tmp);
    tmp = nullptr;
    tmp_bytes = 0;
    GRE_CUDA(cudaMalloc(&tmp, bytes));
    tmp_bytes = bytes;
    return GRE_SUCCESS;
  }
  int reserve(uint64_t need, cudaStream_t s) {
    if (need <= cap) return GRE_SUCCESS;
    const uint64_t ncap = std::max<uint64_t>(need, cap + cap / 2 + 1024);
    uint64_t* ne = nullptr;
    GRE_CUDA(cudaMalloc(&ne, sizeof(uint64_t) * ncap));
    if (m) {
      const cudaError_t e = cudaMemcpyAsync(ne, edges, sizeof(uint64_t) * m, cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) {
        cudaFree(ne);
        return cuda_status(e, "edge list growth", __FILE__, __LINE__);
      }
      GRE_CUDA(cudaStreamSynchronize(s));
    }
    cudaFree(edges);
    edges = ne;
    cap = ncap;
    return GRE_SUCCESS;
  }
};

// Stage A (asynchronous): the chunk's bytes to the device and the positions of its lines.
int chunk_begin(gre_graph g, Ingest& in, const char* host, uint64_t len) {
  cudaStream_t s = g->stream;
  GRE_CUDA(cudaMemcpyAsync(in.dbuf, host, len, cudaMemcpyHostToDevice, s));
  cub::CountingInputIterator<uint32_t> pos(0);
  size_t tb = 0;
  cub::DeviceSelect::If(nullptr, tb, pos, in.starts, in.counters, (int64_t)len, LineStart{in.dbuf}, s);
  GRE_CHECK(in.scratch(tb));
  GRE_CUDA(cub::DeviceSelect::If(in.tmp, tb, pos, in.starts, in.counters, (int64_t)len, LineStart{in.dbuf}, s));
  return GRE_SUCCESS;
}

// Stage B: parse every line, append the valid edges in order.  On a bad line returns its code
// and global line index (earlier chunks were clean, so it is the first in file order).
int chunk_end(gre_graph g, Ingest& in, uint64_t len, uint64_t line0, uint64_t nv, uint64_t* nlines_out, uint64_t* bad_line) {
  cudaStream_t s = g->stream;
  uint64_t nlines = 0;
  GRE_CUDA(cudaMemcpyAsync(&nlines, in.counters, sizeof nlines, cudaMemcpyDeviceToHost, s));
  GRE_CUDA(cudaStreamSynchronize(s));
  *nlines_out = nlines;
  if (!nlines) return GRE_SUCCESS;
  k_parse_lines<<<grid_for(nlines, 256), 256, 0, s>>>(in.dbuf, len, in.starts, nlines, line0, nv, in.parsed, in.counters + 2);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(in.reserve(in.m + nlines, s));
  size_t tb = 0;
  cub::DeviceSelect::If(nullptr, tb, in.parsed, in.edges + in.m, in.counters + 1, (int64_t)nlines, NotSkip{}, s);
  GRE_CHECK(in.scratch(tb));
  GRE_CUDA(cub::DeviceSelect::If(in.tmp, tb, in.parsed, in.edges + in.m, in.counters + 1, (int64_t)nlines, NotSkip{}, s));
  unsigned long long h[2] = {0, 0};
  GRE_CUDA(cudaMemcpyAsync(h, in.counters + 1, sizeof h, cudaMemcpyDeviceToHost, s));
  GRE_CUDA(cudaStreamSynchronize(s));
  if (h[1] != ~0ull) {
    *bad_line = h[1] >> 4;
    return (int)(h[1] & 15u);
  }
  in.m += h[0];
  return GRE_SUCCESS;
}

// Fills buf after `carry` bytes already there; sets *len (bytes held), *cut (end of the last
// whole line) and *eof.  A last line without '\n' gets one (it is still a line).
int fill(FILE* f, char* buf, uint64_t chunk, uint64_t carry, uint64_t* len, uint64_t* cut, bool* eof, const std::string& name) {
  const size_t got = fread(buf + carry, 1, chunk - carry, f);
  *len = carry + got;
  *eof = got < chunk - carry;
  *cut = 0;
  if (*len == 0) return GRE_SUCCESS;
  if (*eof) {
    if (buf[*len - 1] != '\n') buf[(*len)++] = '\n';
    *cut = *len;
    return GRE_SUCCESS;
  }
  for (uint64_t i = *len; i > 0; --i)
    if (buf[i - 1] == '\n') {
      *cut = i;
      return GRE_SUCCESS;
    }
  set_error("%s: a line longer than the ingest chunk (%llu bytes)", name.c_str(), (unsigned long long)chunk);
  return GRE_IO_ERROR;
}

// Streams one file through the two pinned buffers: while the device copies and scans chunk k,
// the host reads chunk k+1 into the other buffer.  *missing is set (and nothing else done) when
// the file cannot be opened: the caller decides whether that ends the file list.
int ingest_file(gre_graph g, Ingest& in, const std::string& name, uint64_t chunk, uint64_t nv, uint64_t* line0,
                bool* missing) {
  FILE* f = fopen(name.c_str(), "rb");
  *missing = !f;
  if (!f) return GRE_SUCCESS;
  const uint64_t file_line0 = *line0;
  int cur = 0;
  uint64_t len = 0, cut = 0;
  bool eof = false;
  int st = fill(f, in.pin[cur], chunk, 0, &len, &cut, &eof, name);
  while (!st && cut > 0) {
    st = chunk_begin(g, in, in.pin[cur], cut);
    if (st) break;
    // the partial last line moves to the other buffer, which the next read fills after it
    const uint64_t carry = len - cut;
    if (carry) memcpy(in.pin[cur ^ 1], in.pin[cur] + cut, carry);
    uint64_t nlen = 0, ncut = 0;
    bool neof = true;
    int rst = GRE_SUCCESS;
    if (!eof) rst = fill(f, in.pin[cur ^ 1], chunk, carry, &nlen, &ncut, &neof, name);
    uint64_t nlines = 0, bad = 0;
    st = chunk_end(g, in, cut, *line0, nv, &nlines, &bad);
    if (st == GRE_IO_ERROR || st == GRE_INVALID_ARG)
      set_error("%s:%llu: expected \"u v\" with u, v < n = %llu", name.c_str(), (unsigned long long)(bad - file_line0 + 1),
                (unsigned long long)nv);
    if (!st) st = rst;
    *line0 += nlines;
    cur ^= 1;
    len = nlen;
    cut = ncut;
    eof = neof;
  }
  fclose(f);
  return st;
}

}  // namespace

namespace {

int read_meta(const char* prefix, uint64_t* nv, uint64_t* ne) {
  const std::string meta = std::string(prefix) + ".meta";
  FILE* f = fopen(meta.c_str(), "r");
  if (!f) {
    set_error("cannot open %s", meta.c_str());
    return GRE_IO_ERROR;
  }
  unsigned long long a = 0, b = 0;
  const int k = fscanf(f, "%llu %llu", &a, &b);
  fclose(f);
  if (k != 2) {
    set_error("%s: expected \"n m\"", meta.c_str());
    return GRE_IO_ERROR;
  }
  if (a == 0 || a > 0xffffffffull) {
    set_error("%s: vertex count %llu out of range", meta.c_str(), a);
    return GRE_INVALID_ARG;
  }
  *nv = a;
  *ne = b;
  return GRE_SUCCESS;
}

int alloc_ingest(gre_graph g, Ingest& in, uint64_t chunk, uint64_t ne) {
  GRE_CUDA(cudaHostAlloc((void**)&in.pin[0], chunk + 1, cudaHostAllocDefault));
  GRE_CUDA(cudaHostAlloc((void**)&in.pin[1], chunk + 1, cudaHostAllocDefault));
  GRE_CUDA(cudaMalloc(&in.dbuf, chunk + 1));
  GRE_CUDA(cudaMalloc(&in.starts, sizeof(uint32_t) * (chunk + 1)));
  GRE_CUDA(cudaMalloc(&in.parsed, sizeof(uint64_t) * (chunk + 1)));
  GRE_CUDA(cudaMalloc(&in.counters, sizeof(unsigned long long) * 3));
  GRE_CUDA(cudaMemsetAsync(in.counters + 2, 0xff, sizeof(unsigned long long), g->stream));
  return in.reserve(ne ? ne : 1024, g->stream);
}

// The edge list (packed source << 32 | target, in file order) -> CSR of g: a stable sort by
// source keeps file order within a source (GraphInCSR::build); then relabelling and the
// derived arrays.
int finish_ingest(gre_graph g, Ingest& in, uint64_t nv, uint32_t flags) {
  const uint64_t m = in.m;
  g->n = nv;
  g->m = m;
  GRE_CUDA(cudaMalloc(&g->off, sizeof(uint64_t) * (nv + 1)));
  GRE_CUDA(cudaMalloc(&g->col, sizeof(uint32_t) * (m ? m : 1)));
  if (m) {
    uint64_t* alt = nullptr;
    GRE_CUDA(cudaMalloc(&alt, sizeof(uint64_t) * m));
    cub::DoubleBuffer<uint64_t> dk(in.edges, alt);
    int bits = 1;
    while (bits < 32 && (1ull << bits) < nv) ++bits;
    size_t tb = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, dk, m, 32, 32 + bits, g->stream);
    int st = in.scratch(tb);
    cudaError_t e = cudaSuccess;
    if (!st) e = cub::DeviceRadixSort::SortKeys(in.tmp, tb, dk, m, 32, 32 + bits, g->stream);
    if (!st && e == cudaSuccess) {
      k_split_packed<<<grid_for(m, 256), 256, 0, g->stream>>>(m, dk.Current(), g->col);
      k_offsets_by_high<<<grid_for(nv + 1, 256), 256, 0, g->stream>>>(nv, m, dk.Current(), g->off);
      e = cudaStreamSynchronize(g->stream);
    }
    if (dk.Current() == alt) {  // keep `in` owning exactly one of the two buffers
      cudaFree(in.edges);
      in.edges = alt;
    } else {
      cudaFree(alt);
    }
    if (st) return st;
    if (e != cudaSuccess) return cuda_status(e, "edge sort", __FILE__, __LINE__);
  } else {
    GRE_CUDA(cudaMemsetAsync(g->off, 0, sizeof(uint64_t) * (nv + 1), g->stream));
  }
  // release the parse buffers before the derived arrays are built
  {
    Ingest done;
    std::swap(done.pin[0], in.pin[0]);
    std::swap(done.pin[1], in.pin[1]);
    std::swap(done.dbuf, in.dbuf);
    std::swap(done.starts, in.starts);
    std::swap(done.parsed, in.parsed);
    std::swap(done.edges, in.edges);
    std::swap(done.tmp, in.tmp);
  }
  if (flags & GRE_GRAPH_REORDER) GRE_CHECK(reorder_graph(g));
  return finish_graph(g);
}

// (source, target) pairs of 64-bit vertex ids -> packed 32-bit pairs; ids not below n flag
// GRE_INVALID_ARG with the pair index (the first bad pair in file order decides).
__global__ void k_pack_pairs(const unsigned long long* __restrict__ pairs, uint64_t count, uint64_t pair0, uint64_t nv,
                             uint64_t* __restrict__ out, unsigned long long* __restrict__ first_err) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long u = pairs[2 * i], v = pairs[2 * i + 1];
    if (u >= nv || v >= nv) {
      atomicMin(first_err, (unsigned long long)(((pair0 + i) << 4) | (uint64_t)GRE_INVALID_ARG));
      out[i] = 0;
    } else {
      out[i] = (u << 32) | v;
    }
  }
}

}  // namespace

int device_ingest(const char* prefix, uint32_t flags, int device, gre_graph* out) {
  uint64_t nv = 0, ne = 0;
  GRE_CHECK(read_meta(prefix, &nv, &ne));
  gre_graph g = nullptr;
  GRE_CHECK(new_graph(device, flags, &g));
  GraphGuard guard{g};
  Ingest in;
  const uint64_t chunk = chunk_bytes();
  GRE_CHECK(alloc_ingest(g, in, chunk, ne));
  uint64_t line0 = 0;
  for (int i = 0;; ++i) {
    const std::string name = std::string(prefix) + ".edges." + std::to_string(i);
    bool missing = false;
    const int st = ingest_file(g, in, name, chunk, nv, &line0, &missing);
    if (st) return st;
    if (missing) {
      if (i > 0) break;  // the files are .edges.0 .. .edges.<P-1>
      set_error("cannot open %s", name.c_str());
      return GRE_IO_ERROR;
    }
  }
  GRE_CHECK(finish_ingest(g, in, nv, flags));
  *out = guard.release();
  return GRE_SUCCESS;
}

// The reference's saved partitions (GraphIngress::loadEdgePartitions, GraphIngress.hpp:
// 1024-1071): <prefix>.part.<P>.<r> holds rank r's edges as binary (vid_t, vid_t) pairs.  One
// GPU holds every rank's part: the P files are read in rank order into one edge list (the
// .outdegree and .scatterMap files only serve the rank exchange and are not needed).
int device_ingest_parts(const char* prefix, uint32_t nparts, uint32_t flags, int device, gre_graph* out) {
  uint64_t nv = 0, ne = 0;
  GRE_CHECK(read_meta(prefix, &nv, &ne));
  if (nparts == 0) {
    set_error("gre_graph_load_parts: zero parts");
    return GRE_INVALID_ARG;
  }
  gre_graph g = nullptr;
  GRE_CHECK(new_graph(device, flags, &g));
  GraphGuard guard{g};
  Ingest in;
  const uint64_t chunk = (chunk_bytes() / 16) * 16 ? (chunk_bytes() / 16) * 16 : 16;  // whole pairs
  GRE_CHECK(alloc_ingest(g, in, chunk, ne));
  uint64_t pair0 = 0;
  for (uint32_t r = 0; r < nparts; ++r) {
    const std::string name = std::string(prefix) + ".part." + std::to_string(nparts) + "." + std::to_string(r);
    FILE* f = fopen(name.c_str(), "rb");
    if (!f) {
      set_error("cannot open %s", name.c_str());
      return GRE_IO_ERROR;
    }
    int st = GRE_SUCCESS;
    const uint64_t file_pair0 = pair0;
    for (;;) {
      const size_t got = fread(in.pin[0], 1, chunk, f);
      if (got % 16) {
        set_error("%s: size is not a multiple of 16 bytes (vid_t pairs)", name.c_str());
        st = GRE_IO_ERROR;
        break;
      }
      const uint64_t cnt = got / 16;
      if (cnt) {
        cudaError_t e = cudaMemcpyAsync(in.dbuf, in.pin[0], got, cudaMemcpyHostToDevice, g->stream);
        if (e == cudaSuccess) st = in.reserve(in.m + cnt, g->stream);
        if (e == cudaSuccess && !st) {
          k_pack_pairs<<<grid_for(cnt, 256), 256, 0, g->stream>>>((const unsigned long long*)in.dbuf, cnt, pair0, nv, in.edges + in.m,
                                                                  in.counters + 2);
          unsigned long long bad = 0;
          e = cudaMemcpyAsync(&bad, in.counters + 2, sizeof bad, cudaMemcpyDeviceToHost, g->stream);
          if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
          if (e == cudaSuccess && bad != ~0ull) {
            set_error("%s: pair %llu has a vertex id not below n = %llu", name.c_str(), (unsigned long long)((bad >> 4) - file_pair0),
                      (unsigned long long)nv);
            st = GRE_INVALID_ARG;
          }
        }
        if (e != cudaSuccess && !st) st = cuda_status(e, "partition read", __FILE__, __LINE__);
        if (st) break;
        in.m += cnt;
        pair0 += cnt;
      }
      if (got < chunk) break;
    }
    fclose(f);
    if (st) return st;
  }
  GRE_CHECK(finish_ingest(g, in, nv, flags));
  *out = guard.release();
  return GRE_SUCCESS;
}

}  // namespace gre
