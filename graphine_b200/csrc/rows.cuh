// Degree-binned row reductions over a CSR or CSC: the pull form of the superstep's
// scatter+combine for sums (PageRank, weighted PageRank, its adjoint).
//
// Rows are grouped once per graph by degree (DegreeBins, schedule chosen by the autotuner in
// bins.cu): bins 0..5 give a row 1, 2, 4, 8, 16 or 32 lanes (by default degree 1-4, 5-8, 9-16,
// 17-32, 33-64, 65-4096: about four arcs per lane per pass); bin 6 gives a row one CTA (by
// default 4097-65536); bin 7 splits a row into chunks of hub_chunk arcs (65536), one CTA each,
// whose partial sums are added in chunk order by a second kernel.  Lane j of a group adds arcs
// j, j+L, j+2L, ... (four independent loads per pass) and the group reduces with xor shuffles,
// so every row's sum has a fixed association order for a given schedule: results are
// deterministic run to run.  Column indices of one group are contiguous (coalesced); the
// gathered value is the only random access.
//
//   Gather: __device__ double operator()(uint32_t row, uint64_t arc) const   value of one arc
//   Finish: __device__ void operator()(uint32_t row, double sum) const
#pragma once
#include "gre_internal.cuh"

namespace gre {
namespace rows {

constexpr int kCta = 256;

// Sum of gat(v, a) over a = a0 + lig, a0 + lig + L, ... < a1.  Four arcs per pass so that each
// lane has four independent (column, gathered value) load chains in flight: the loop is bound
// by memory latency, not bandwidth, when a lane waits on one chain at a time.
template <int L, class Gather>
__device__ __forceinline__ double strided_sum(Gather& gat, uint32_t v, uint64_t a0, uint64_t a1, uint32_t lig) {
  double acc = 0.0;
  uint64_t a = a0 + lig;
  for (; a + 3 * (uint64_t)L < a1; a += 4 * (uint64_t)L) {
    const double x0 = gat(v, a), x1 = gat(v, a + L), x2 = gat(v, a + 2 * L), x3 = gat(v, a + 3 * L);
    acc += x0;
    acc += x1;
    acc += x2;
    acc += x3;
  }
  for (; a < a1; a += L) acc += gat(v, a);
  return acc;
}

template <int L, class Gather, class Finish>
__global__ void __launch_bounds__(256) k_rows_lanes(const uint32_t* __restrict__ rows, uint64_t count,
                                                     const uint64_t* __restrict__ off, Gather gat, Finish fin) {
  constexpr int G = 32 / L;  // groups per warp
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lig = lane % L;
  const uint64_t warp = tid >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t base = warp * G; base < count; base += nwarps * G) {
    const uint64_t i = base + lane / L;
    const bool valid = i < count;
    double acc = 0.0;
    uint32_t v = 0;
    if (valid) {
      v = rows[i];
      acc = strided_sum<L>(gat, v, off[v], off[v + 1], lig);
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (valid && lig == 0) fin(v, acc);
  }
}

__device__ __forceinline__ double block_sum(double x, double* smem) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) smem[w] = x;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += smem[i];
  }
  __syncthreads();
  return t;  // valid in thread 0
}

template <class Gather, class Finish>
__global__ void __launch_bounds__(kCta) k_rows_cta(const uint32_t* __restrict__ rows, uint64_t count,
                                                    const uint64_t* __restrict__ off, Gather gat, Finish fin) {
  __shared__ double smem[kCta / 32];
  for (uint64_t i = blockIdx.x; i < count; i += gridDim.x) {
    const uint32_t v = rows[i];
    double acc = strided_sum<kCta>(gat, v, off[v], off[v + 1], threadIdx.x);
    acc = block_sum(acc, smem);
    if (threadIdx.x == 0) fin(v, acc);
  }
}

template <class Gather>
__global__ void __launch_bounds__(kCta) k_rows_chunks(const uint32_t* __restrict__ rows, const uint64_t* __restrict__ chunk_row,
                                                       const uint64_t* __restrict__ chunk_begin, uint64_t nchunks, uint64_t chunk,
                                                       const uint64_t* __restrict__ off, Gather gat, double* __restrict__ partial) {
  __shared__ double smem[kCta / 32];
  for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const uint32_t v = rows[chunk_row[c]];
    const uint64_t a0 = chunk_begin[c];
    const uint64_t end = off[v + 1];
    const uint64_t a1 = (a0 + chunk < end) ? a0 + chunk : end;
    double acc = strided_sum<kCta>(gat, v, a0, a1, threadIdx.x);
    acc = block_sum(acc, smem);
    if (threadIdx.x == 0) partial[c] = acc;
  }
}

// Window-split rows (DegreeBins::seg_*): CTA per chunk in processing order, partial sums by slot.
template <class Gather>
__global__ void __launch_bounds__(kCta) k_rows_seg(const uint32_t* __restrict__ row, const uint64_t* __restrict__ begin,
                                                   const uint64_t* __restrict__ end, const uint64_t* __restrict__ slot,
                                                   uint64_t nchunks, Gather gat, double* __restrict__ partial) {
  __shared__ double smem[kCta / 32];
  for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const uint32_t v = row[c];
    double acc = strided_sum<kCta>(gat, v, begin[c], end[c], threadIdx.x);
    acc = block_sum(acc, smem);
    if (threadIdx.x == 0) partial[slot[c]] = acc;
  }
}

template <class Finish>
__global__ void k_rows_seg_finish(const uint32_t* __restrict__ rows, uint64_t count, const uint64_t* __restrict__ first,
                                  const double* __restrict__ partial, Finish fin) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint64_t c = first[i]; c < first[i + 1]; ++c) s += partial[c];
    fin(rows[i], s);
  }
}

template <class Finish>
__global__ void k_rows_chunk_finish(const uint32_t* __restrict__ rows, uint64_t count, const uint64_t* __restrict__ first,
                                    const double* __restrict__ partial, Finish fin) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint64_t c = first[i]; c < first[i + 1]; ++c) s += partial[c];
    fin(rows[i], s);
  }
}

// Launch the reductions of every non-empty row.  `partial` holds bins.n_partials doubles.
template <class Gather, class Finish>
int reduce_rows(const DegreeBins& B, const uint64_t* off, Gather gat, Finish fin, double* partial, cudaStream_t s) {
  const uint32_t* r = B.rows;
  auto grid = [](uint64_t threads) { return grid_for(threads, 256, 8); };
  if (B.count[0]) k_rows_lanes<1><<<grid(B.count[0]), 256, 0, s>>>(r + B.start[0], B.count[0], off, gat, fin);
  if (B.count[1]) k_rows_lanes<2><<<grid(B.count[1] * 2), 256, 0, s>>>(r + B.start[1], B.count[1], off, gat, fin);
  if (B.count[2]) k_rows_lanes<4><<<grid(B.count[2] * 4), 256, 0, s>>>(r + B.start[2], B.count[2], off, gat, fin);
  if (B.count[3]) k_rows_lanes<8><<<grid(B.count[3] * 8), 256, 0, s>>>(r + B.start[3], B.count[3], off, gat, fin);
  if (B.count[4]) k_rows_lanes<16><<<grid(B.count[4] * 16), 256, 0, s>>>(r + B.start[4], B.count[4], off, gat, fin);
  if (B.count[5]) k_rows_lanes<32><<<grid(B.count[5] * 32), 256, 0, s>>>(r + B.start[5], B.count[5], off, gat, fin);
  if (B.seg_nchunks) {  // rows above cta_min, window by window
    k_rows_seg<<<grid_for(B.seg_nchunks * kCta, kCta, 8), kCta, 0, s>>>(B.seg_row, B.seg_begin, B.seg_end, B.seg_slot,
                                                                         B.seg_nchunks, gat, partial);
    k_rows_seg_finish<<<grid_for(B.seg_nrows, 128, 4), 128, 0, s>>>(B.seg_rows, B.seg_nrows, B.seg_first, partial, fin);
    GRE_LAUNCH_CHECK();
    return GRE_SUCCESS;
  }
  if (B.count[6]) k_rows_cta<<<grid_for(B.count[6] * kCta, kCta, 8), kCta, 0, s>>>(r + B.start[6], B.count[6], off, gat, fin);
  if (B.count[7]) {
    k_rows_chunks<<<grid_for(B.n_hub_chunks * kCta, kCta, 8), kCta, 0, s>>>(r + B.start[7], B.hub_chunk_row, B.hub_chunk_begin,
                                                                            B.n_hub_chunks, B.sched.hub_chunk, off, gat, partial);
    k_rows_chunk_finish<<<grid_for(B.count[7], 128, 4), 128, 0, s>>>(r + B.start[7], B.count[7], B.hub_chunk_first, partial, fin);
  }
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

// Number of non-empty rows of the bins (for byte models).
inline uint64_t nonempty_rows(const DegreeBins& B) {
  uint64_t s = 0;
  for (int i = 0; i < DegreeBins::NB; ++i) s += B.count[i];
  return s;
}

}  // namespace rows
}  // namespace gre
