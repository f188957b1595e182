// gre/vertex_code.cuh — device-side VertexCode plugin concept and the generic superstep engine.
//
// A plugin is a struct passed by value to the kernels (device pointers + scalars) with the
// callbacks of GRE::VertexCode (include/VertexCode/VertexCode.hpp:25-63), same names, same
// return-value meaning:
//
//   typedef ... msg_t;                                          // scatter/combine data type
//   __device__ bool init(uint32_t lv);                          // true: lv starts active
//   template <class Ctx> __device__ void scatter(Ctx& ctx, uint32_t lsrc, uint32_t ldst,
//                                                uint64_t arc);  // calls ctx.sendMessage
//   __device__ bool combine(uint32_t ldst, const msg_t& msg);   // true: ldst gets applied
//   __device__ bool apply(uint32_t lv);                         // true: lv becomes active
//   __device__ bool assert_to_halt(uint32_t lv);                // true: lv leaves the frontier
//   void reduce();                                              // host, once per superstep
//   void output_statistics(const EngineContext&);               // host, once after the run
//                                                               // (optional)
//
// The reference's combine receives a striped spin lock (Util/vLock.hpp:75-99); on the device
// combine is written with atomics (atomicAdd / atomicMin / atomicCAS) and takes no lock.
// `arc` is the CSR arc id for out-arcs and the CSR id of the same arc for in-arcs when the
// graph has an arc map (otherwise the CSC slot), in place of the reference's edge iterator.
//
// SynchronousEngine<VC>::run<dir> executes SynchronousEngine::run_master/fn_worker_tp
// (include/Engine/Engine.hpp:247-406, 423-814) at one rank:
//   init(all or sources) -> repeat { compute: every active vertex scatters along its arcs,
//   sendMessage = combine + set nextSet bit; assert_to_halt clears the active bit | apply:
//   for each nextSet bit, apply() true sets the active bit | rebuild the active list |
//   reduce() | stop when the list is empty or after max supersteps }.
// The frontier is a 32-bit-word bitmap plus a compacted vertex list; the apply kernel builds
// each active-bitmap word with one warp ballot (32 consecutive vertices per warp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>
#include <vector>

namespace gre {

enum VcDir { VC_OUT = 0, VC_IN = 1, VC_INOUT = 2 };

// Read-only view of a device graph (CSR = out-arcs, CSC = in-arcs).
struct DeviceGraphView {
  uint64_t n;
  const uint64_t* off;
  const uint32_t* col;
  const uint64_t* roff;
  const uint32_t* rcol;
  const uint64_t* rarc;  // may be null
};

// Context handed to scatter: ctx.sendMessage(ldst, msg) is SynchronousEngine::sendMessage
// (Engine.hpp:1384-1389): combine, and on success test-and-set the nextSet bit.
template <class VC>
struct SendCtx {
  VC& vc;
  uint32_t* next_bits;
  __device__ __forceinline__ void sendMessage(uint32_t ldst, const typename VC::msg_t& msg) {
    if (vc.combine(ldst, msg)) {
      const uint32_t bit = 1u << (ldst & 31u);
      uint32_t* w = next_bits + (ldst >> 5);
      if (!(*(volatile uint32_t*)w & bit)) atomicOr(w, bit);
    }
  }
};

// What the engine hands output_statistics (the reference passes its DistributedContext,
// VertexCode.hpp:68-70): the stream the run used and the run's counters.
struct EngineContext {
  cudaStream_t stream;
  uint64_t n;
  long supersteps;
  uint64_t arcs_scanned;
};

namespace vc_detail {

// output_statistics is optional, as in the reference (VertexCode.hpp:68-70 is an empty default)
template <class VC, class = void>
struct has_output_statistics : std::false_type {};
template <class VC>
struct has_output_statistics<VC, std::void_t<decltype(std::declval<VC&>().output_statistics(
                                     std::declval<const EngineContext&>()))>> : std::true_type {};

template <class VC>
__global__ void k_init_all(VC vc, uint64_t n, uint32_t* curr_bits) {
  const uint64_t nwords = (n + 31) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = warp; w < nwords; w += nwarps) {
    const uint64_t v = (w << 5) + lane;
    bool act = false;
    if (v < n) act = vc.init((uint32_t)v);
    const uint32_t ball = __ballot_sync(0xffffffffu, act);
    if (lane == 0) curr_bits[w] = ball;
  }
}

// Sources in order, by one thread (the reference does this on worker 0, Engine.hpp:459-471).
template <class VC>
__global__ void k_init_set(VC vc, const uint32_t* srcs, uint32_t nsrc, uint32_t* curr_bits) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (uint32_t i = 0; i < nsrc; ++i) {
    const uint32_t v = srcs[i];
    if (vc.init(v)) curr_bits[v >> 5] |= 1u << (v & 31u);
  }
}

// Active bitmap -> list; also sums the degrees of the listed vertices (arcs to scan).
__global__ void k_compact(uint64_t n, const uint32_t* __restrict__ bits, uint32_t* __restrict__ list,
                          uint32_t* __restrict__ count, const uint64_t* __restrict__ off,
                          const uint64_t* __restrict__ roff, int dir, unsigned long long* __restrict__ arcs) {
  const uint64_t nwords = (n + 31) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = tid - lane; base < nwords; base += nthreads) {
    const uint64_t w = base + lane;
    const uint32_t word = (w < nwords) ? bits[w] : 0u;
    const uint32_t c = __popc(word);
    uint32_t incl = c;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t pos = 0;
    if (lane == 31 && total) pos = atomicAdd(count, total);
    pos = __shfl_sync(0xffffffffu, pos, 31) + incl - c;
    unsigned long long deg = 0;
    uint32_t x = word;
    while (x) {
      const uint32_t b = __ffs(x) - 1;
      x &= x - 1;
      const uint32_t v = (uint32_t)(w << 5) + b;
      list[pos++] = v;
      if (dir != VC_IN) deg += off[v + 1] - off[v];
      if (dir != VC_OUT) deg += roff[v + 1] - roff[v];
    }
    for (int o = 16; o > 0; o >>= 1) deg += __shfl_xor_sync(0xffffffffu, deg, o);
    if (lane == 0 && deg) atomicAdd(arcs, deg);
  }
}

// Compute phase: one warp per active vertex, lanes stride over its arcs.
template <class VC, int DIR>
__global__ void k_compute(VC vc, DeviceGraphView g, const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                          uint32_t* __restrict__ curr_bits, uint32_t* __restrict__ next_bits) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t cnt = *count;
  SendCtx<VC> ctx{vc, next_bits};
  for (uint64_t i = warp; i < cnt; i += nwarps) {
    const uint32_t u = list[i];
    if (DIR == VC_OUT || DIR == VC_INOUT) {
      const uint64_t a1 = g.off[u + 1];
      for (uint64_t a = g.off[u] + lane; a < a1; a += 32) vc.scatter(ctx, u, g.col[a], a);
    }
    if (DIR == VC_IN || DIR == VC_INOUT) {
      const uint64_t a1 = g.roff[u + 1];
      for (uint64_t a = g.roff[u] + lane; a < a1; a += 32) vc.scatter(ctx, u, g.rcol[a], g.rarc ? g.rarc[a] : a);
    }
    __syncwarp();
    if (lane == 0 && vc.assert_to_halt(u)) atomicAnd(curr_bits + (u >> 5), ~(1u << (u & 31u)));
  }
}

// Apply phase: warp w handles bitmap word w (32 consecutive vertices).
template <class VC>
__global__ void k_apply(VC vc, uint64_t n, const uint32_t* __restrict__ next_bits, uint32_t* __restrict__ curr_bits) {
  const uint64_t nwords = (n + 31) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = warp; w < nwords; w += nwarps) {
    const uint32_t nb = next_bits[w];
    if (!nb) continue;  // uniform per warp
    const uint64_t v = (w << 5) + lane;
    bool act = false;
    if (((nb >> lane) & 1u) && v < n) act = vc.apply((uint32_t)v);
    const uint32_t ball = __ballot_sync(0xffffffffu, act);
    if (lane == 0 && ball) curr_bits[w] |= ball;
  }
}

}  // namespace vc_detail

// Device scratch the engine needs for a graph of n vertices.
inline size_t vc_scratch_bytes(uint64_t n) {
  const uint64_t nwords = (n + 31) >> 5;
  return 2 * nwords * sizeof(uint32_t) + n * sizeof(uint32_t) + 64;
}

// SourceVertexSet (Graph/VertexSet.hpp:286-347): all vertices, or a list of sources.
struct SourceSet {
  bool all = false;
  const uint32_t* dev_vertices = nullptr;  // device array
  uint32_t count = 0;
};

template <class VC>
class SynchronousEngine {
 public:
  // scratch: device memory of vc_scratch_bytes(g.n) bytes, owned by the caller.
  SynchronousEngine(const DeviceGraphView& g, VC& vc, cudaStream_t stream, void* scratch)
      : g_(g), vc_(vc), stream_(stream) {
    const uint64_t nwords = (g.n + 31) >> 5;
    char* p = (char*)scratch;
    curr_bits_ = (uint32_t*)p;
    p += nwords * sizeof(uint32_t);
    next_bits_ = (uint32_t*)p;
    p += nwords * sizeof(uint32_t);
    list_ = (uint32_t*)p;
    p += g.n * sizeof(uint32_t);
    counters_ = (uint32_t*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
  }
  // SynchronousEngine::configMaxSupersteps (Engine.hpp:148-153)
  void configMaxSupersteps(long n) { max_supersteps_ = n > 0 ? n : 1024; }
  // SynchronousEngine::getSuperstepCount (Engine.hpp:1307-1309)
  long getSuperstepCount() const { return superstep_; }
  const std::vector<uint64_t>& activeCounts() const { return active_; }
  uint64_t arcsScanned() const { return arcs_; }

  // SynchronousEngine::run<dir> (Engine.hpp:180-202).  Returns a cudaError_t.
  template <int DIR>
  cudaError_t run(const SourceSet& src, int sms) {
    using namespace vc_detail;
    const uint64_t n = g_.n;
    const uint64_t nwords = (n + 31) >> 5;
    const int blk = 256;
    const int grid_words = (int)(((nwords * 32 + blk - 1) / blk) < (uint64_t)sms * 8 ? ((nwords * 32 + blk - 1) / blk) : (uint64_t)sms * 8);
    const int grid = grid_words > 0 ? grid_words : 1;
    active_.clear();
    arcs_ = 0;
    superstep_ = 0;
    cudaMemsetAsync(curr_bits_, 0, nwords * sizeof(uint32_t), stream_);
    if (src.all) k_init_all<VC><<<grid, blk, 0, stream_>>>(vc_, n, curr_bits_);
    else k_init_set<VC><<<1, 32, 0, stream_>>>(vc_, src.dev_vertices, src.count, curr_bits_);
    cudaError_t e = compact(sms);
    if (e != cudaSuccess) return e;
    uint32_t count = host_count_;
    long ss = 0;
    for (ss = 0; ss < max_supersteps_; ++ss) {
      cudaMemsetAsync(next_bits_, 0, nwords * sizeof(uint32_t), stream_);
      if (count) {
        const uint64_t want_warps = count;
        int cgrid = (int)((want_warps * 32 + blk - 1) / blk);
        if (cgrid > sms * 16) cgrid = sms * 16;
        if (cgrid < 1) cgrid = 1;
        k_compute<VC, DIR><<<cgrid, blk, 0, stream_>>>(vc_, g_, list_, counters_, curr_bits_, next_bits_);
      }
      k_apply<VC><<<grid, blk, 0, stream_>>>(vc_, n, next_bits_, curr_bits_);
      e = compact(sms);
      if (e != cudaSuccess) return e;
      count = host_count_;
      vc_.reduce();
      active_.push_back(count);
      if (count == 0) break;
    }
    superstep_ = ss;
    // run_master calls output_statistics once the loop has ended (Engine.hpp:402-404)
    if constexpr (vc_detail::has_output_statistics<VC>::value) vc_.output_statistics(EngineContext{stream_, n, ss, arcs_});
    return cudaGetLastError();
  }

 private:
  cudaError_t compact(int sms) {
    const uint64_t nwords = (g_.n + 31) >> 5;
    cudaMemsetAsync(counters_, 0, 16, stream_);
    int grid = (int)((nwords + 255) / 256);
    if (grid > sms * 8) grid = sms * 8;
    if (grid < 1) grid = 1;
    vc_detail::k_compact<<<grid, 256, 0, stream_>>>(g_.n, curr_bits_, list_, counters_, g_.off, g_.roff, dir_for_arcs_,
                                                    (unsigned long long*)(counters_ + 2));
    uint32_t h[4];
    cudaError_t e = cudaMemcpyAsync(h, counters_, sizeof h, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return e;
    host_count_ = h[0];
    arcs_ += ((uint64_t)h[3] << 32) | h[2];
    return cudaSuccess;
  }

 public:
  int dir_for_arcs_ = VC_OUT;  // which arcs the compact kernel sums for arcsScanned()

 private:
  DeviceGraphView g_;
  VC& vc_;
  cudaStream_t stream_;
  uint32_t *curr_bits_, *next_bits_, *list_, *counters_;
  long max_supersteps_ = 1024;
  long superstep_ = 0;
  uint32_t host_count_ = 0;
  uint64_t arcs_ = 0;
  std::vector<uint64_t> active_;
};

}  // namespace gre
