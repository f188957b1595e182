// PageRank fast paths (FP64, pull over in-arcs):
//   gre_pagerank           one superstep = one degree-binned pull over the CSC
//   gre_ppr                personalised PageRank, looped or batched (128 vectors per pass)
//   gre_pagerank_weighted  weighted forward to a tolerance
//   gre_pagerank_adjoint   implicit adjoint (transposed fixed point) + gradients
//
// The reference superstep (Engine.hpp:592-625 + PageRank.hpp:51-74) pushes pr_scatter[u] along
// every out-arc and adds it into pr_combine[v] under a spin lock, then applies
// pr = 0.15 + 0.85*pr_combine to every vertex that received a message.  The pull form computes
// the same sum per vertex without atomics: pr[v] = tele + d * sum_{u->v} contrib[u], where
// contrib[u] = pr_scatter[u] (0.15/outdeg for the reference variant, pr/outdeg for the power
// iteration).  Vertices without in-arcs receive no message and keep their init value, exactly
// as in the reference (apply is never called for them).
//
// HBM bytes per superstep (algorithmic): 8(n+1) offsets + 4m columns + 8m gathered contrib
// + 4n outdeg + 16n (pr and contrib writes) = 8(n+1) + 12m + 20n.
#include <algorithm>
#include <memory>

#include "gre_internal.cuh"
#include "rows.cuh"

namespace gre {

// ---------------------------------------------------------------------------------------------
// plain PageRank
// ---------------------------------------------------------------------------------------------
struct GatherContrib {
  const uint32_t* __restrict__ rcol;
  const double* __restrict__ contrib;
  // contrib is read-only during a superstep (the next values go to the other buffer)
  __device__ __forceinline__ double operator()(uint32_t, uint64_t a) const { return __ldg(contrib + __ldg(rcol + a)); }
};

struct FinishPR {
  double* __restrict__ pr;
  double* __restrict__ contrib_next;  // null: scatter value never refreshed (reference variant)
  const uint32_t* __restrict__ outdeg;
  double tele, d;
  __device__ __forceinline__ void operator()(uint32_t v, double sum) const {
    const double x = tele + d * sum;
    pr[v] = x;
    if (contrib_next) {
      const uint32_t od = outdeg[v];
      contrib_next[v] = od ? x / (double)od : 0.0;
    }
  }
};

__global__ void k_pr_init(uint64_t n, const uint32_t* __restrict__ outdeg, double tele, double* __restrict__ pr,
                          double* __restrict__ c0, double* __restrict__ c1) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t od = outdeg[v];
    const double c = od ? tele / (double)od : 0.0;
    pr[v] = tele;
    c0[v] = c;
    if (c1) c1[v] = c;
  }
}

static uint64_t pr_bytes_per_iter(uint64_t n, uint64_t m) { return 8 * (n + 1) + 12 * m + 20 * n; }

template <class T>
static int ws_array(gre_graph g, int slot, uint64_t count, T** p) {
  void* v = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &v));
  *p = (T*)v;
  return GRE_SUCCESS;
}

// ---------------------------------------------------------------------------------------------
// personalised PageRank, batched: X[v][k] row-major, one warp per in-arc row, each lane owns
// kCols/32 columns; rows longer than kPprChunk arcs are split into chunks whose partial
// vectors are added in order.
// ---------------------------------------------------------------------------------------------
constexpr int kCols = 128;
constexpr uint64_t kPprChunk = 1024;

__global__ void k_ppr_init(uint64_t n, uint32_t k, const uint32_t* __restrict__ seeds, const uint32_t* __restrict__ outdeg,
                           double tele, double* __restrict__ x, double* __restrict__ c0, double* __restrict__ c1) {
  // zero everything, then place the restart mass
  const uint64_t total = n * kCols;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    x[i] = 0.0;
    c0[i] = 0.0;
    c1[i] = 0.0;
  }
}

__global__ void k_ppr_seed(uint32_t k, const uint32_t* __restrict__ seeds, const uint32_t* __restrict__ outdeg, double tele,
                           double* __restrict__ x, double* __restrict__ c0, double* __restrict__ c1) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
    const uint32_t s = seeds[j];
    const uint32_t od = outdeg[s];
    x[(uint64_t)s * kCols + j] = tele;
    const double c = od ? tele / (double)od : 0.0;
    c0[(uint64_t)s * kCols + j] = c;
    c1[(uint64_t)s * kCols + j] = c;
  }
}

struct PprRow {
  const uint64_t* __restrict__ roff;
  const uint32_t* __restrict__ rcol;
  const double* __restrict__ contrib;
  // adds contrib rows of arcs [a0, a1) into acc (each lane its 4 columns); two arcs per pass
  // keep eight independent loads per lane in flight
  __device__ __forceinline__ void accumulate(uint64_t a0, uint64_t a1, double acc[kCols / 32]) const {
    const uint32_t lane = threadIdx.x & 31u;
    uint64_t a = a0;
    for (; a + 1 < a1; a += 2) {
      const uint32_t u0 = __ldg(rcol + a), u1 = __ldg(rcol + a + 1);
      const double* r0 = contrib + (uint64_t)u0 * kCols + lane;
      const double* r1 = contrib + (uint64_t)u1 * kCols + lane;
      double x0[kCols / 32], x1[kCols / 32];
#pragma unroll
      for (int j = 0; j < kCols / 32; ++j) {
        x0[j] = __ldg(r0 + 32 * j);
        x1[j] = __ldg(r1 + 32 * j);
      }
#pragma unroll
      for (int j = 0; j < kCols / 32; ++j) {
        acc[j] += x0[j];
        acc[j] += x1[j];
      }
    }
    for (; a < a1; ++a) {
      const uint32_t u = __ldg(rcol + a);
      const double* row = contrib + (uint64_t)u * kCols + lane;
#pragma unroll
      for (int j = 0; j < kCols / 32; ++j) acc[j] += __ldg(row + 32 * j);
    }
  }
};

struct PprFinish {
  double* __restrict__ x;
  double* __restrict__ cnext;
  const uint32_t* __restrict__ outdeg;
  const uint32_t* __restrict__ seeds;
  uint32_t k;
  double tele, d;
  __device__ __forceinline__ void operator()(uint32_t v, const double acc[kCols / 32]) const {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t od = outdeg[v];
#pragma unroll
    for (int j = 0; j < kCols / 32; ++j) {
      const uint32_t col = lane + 32 * j;
      const double t = (col < k && seeds[col] == v) ? tele : 0.0;
      const double val = t + d * acc[j];
      x[(uint64_t)v * kCols + col] = val;
      cnext[(uint64_t)v * kCols + col] = od ? val / (double)od : 0.0;
    }
  }
};

// rows of bins 0..4 (degree <= 64): one warp per row
__global__ void __launch_bounds__(256) k_ppr_rows(const uint32_t* __restrict__ rows, uint64_t count, PprRow R, PprFinish F) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = warp; i < count; i += nwarps) {
    const uint32_t v = rows[i];
    double acc[kCols / 32] = {0.0, 0.0, 0.0, 0.0};
    const uint64_t a0 = R.roff[v], a1 = R.roff[v + 1];
    if (a1 - a0 > kPprChunk) continue;  // chunked (uniform: one row per warp)
    R.accumulate(a0, a1, acc);
    F(v, acc);
  }
}

// long rows: chunk c covers arcs [chunk_begin[c], +kPprChunk) of row chunk_row[c]
__global__ void __launch_bounds__(256) k_ppr_chunks(const uint32_t* __restrict__ rows, const uint64_t* __restrict__ chunk_row,
                                                     const uint64_t* __restrict__ chunk_begin, uint64_t nchunks, PprRow R,
                                                     double* __restrict__ partial) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t c = warp; c < nchunks; c += nwarps) {
    const uint32_t v = rows[chunk_row[c]];
    const uint64_t a0 = chunk_begin[c];
    const uint64_t end = R.roff[v + 1];
    const uint64_t a1 = a0 + kPprChunk < end ? a0 + kPprChunk : end;
    double acc[kCols / 32] = {0.0, 0.0, 0.0, 0.0};
    R.accumulate(a0, a1, acc);
#pragma unroll
    for (int j = 0; j < kCols / 32; ++j) partial[c * kCols + lane + 32 * j] = acc[j];
  }
}

__global__ void k_ppr_chunk_finish(const uint32_t* __restrict__ rows, uint64_t count, const uint64_t* __restrict__ first,
                                   const double* __restrict__ partial, PprFinish F) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t i = warp; i < count; i += nwarps) {
    double acc[kCols / 32] = {0.0, 0.0, 0.0, 0.0};
    for (uint64_t c = first[i]; c < first[i + 1]; ++c)
#pragma unroll
      for (int j = 0; j < kCols / 32; ++j) acc[j] += partial[c * kCols + lane + 32 * j];
    F(rows[i], acc);
  }
}

__global__ void k_ppr_transpose(uint64_t n, uint32_t k, const double* __restrict__ x, double* __restrict__ out) {
  // out[j*n + v] = x[v*kCols + j]
  const uint64_t total = (uint64_t)k * n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = i / n, v = i % n;
    out[i] = x[v * kCols + j];
  }
}

struct PprChunks {
  uint64_t nchunks = 0;
  uint64_t* row = nullptr;    // chunk -> index into the long-row list
  uint64_t* begin = nullptr;  // chunk -> first arc
  uint64_t* first = nullptr;  // long row -> first chunk
  uint64_t nrows = 0;
  uint32_t* rows = nullptr;   // long rows (bins 6 and 7, contiguous in the bin list)
};

static int ppr_chunks(gre_graph g, PprChunks* pc) {
  // candidates: rows of more than 64 arcs (bins 5..7, contiguous in the bin list); only those
  // longer than kPprChunk are chunked, the others stay with the warp-per-row kernel
  const DegreeBins& B = g->bins_in;
  const uint64_t cand = B.count[5] + B.count[6] + B.count[7];
  pc->nrows = 0;
  pc->nchunks = 0;
  if (!cand) return GRE_SUCCESS;
  std::vector<uint32_t> rows(cand), lrows;
  std::vector<uint64_t> ho(g->n + 1);
  GRE_CUDA(cudaMemcpy(rows.data(), B.rows + B.start[5], sizeof(uint32_t) * cand, cudaMemcpyDeviceToHost));
  GRE_CUDA(cudaMemcpy(ho.data(), g->roff, sizeof(uint64_t) * (g->n + 1), cudaMemcpyDeviceToHost));
  std::vector<uint64_t> crow, cbeg, first;
  for (uint64_t i = 0; i < cand; ++i) {
    const uint32_t v = rows[i];
    if (ho[v + 1] - ho[v] <= kPprChunk) continue;
    first.push_back(crow.size());
    for (uint64_t a = ho[v]; a < ho[v + 1]; a += kPprChunk) {
      crow.push_back(lrows.size());
      cbeg.push_back(a);
    }
    lrows.push_back(v);
  }
  first.push_back(crow.size());
  pc->nrows = lrows.size();
  pc->nchunks = crow.size();
  if (!pc->nrows) return GRE_SUCCESS;
  void* p;
  GRE_CHECK(g->ws.get(WS_L, sizeof(uint64_t) * (crow.size() * 2 + first.size()) + sizeof(uint32_t) * lrows.size(), &p));
  pc->row = (uint64_t*)p;
  pc->begin = pc->row + crow.size();
  pc->first = pc->begin + crow.size();
  pc->rows = (uint32_t*)(pc->first + first.size());
  GRE_CUDA(cudaMemcpyAsync(pc->row, crow.data(), sizeof(uint64_t) * crow.size(), cudaMemcpyHostToDevice, g->stream));
  GRE_CUDA(cudaMemcpyAsync(pc->begin, cbeg.data(), sizeof(uint64_t) * cbeg.size(), cudaMemcpyHostToDevice, g->stream));
  GRE_CUDA(cudaMemcpyAsync(pc->first, first.data(), sizeof(uint64_t) * first.size(), cudaMemcpyHostToDevice, g->stream));
  GRE_CUDA(cudaMemcpyAsync(pc->rows, lrows.data(), sizeof(uint32_t) * lrows.size(), cudaMemcpyHostToDevice, g->stream));
  GRE_CUDA(cudaStreamSynchronize(g->stream));
  return GRE_SUCCESS;
}

// ---------------------------------------------------------------------------------------------
// single-vector personalised PageRank (looped form): PageRank pull with a one-hot teleport
// ---------------------------------------------------------------------------------------------
struct FinishPPR1 {
  double* __restrict__ x;
  double* __restrict__ cnext;
  const uint32_t* __restrict__ outdeg;
  uint32_t seed;
  double tele, d;
  __device__ __forceinline__ void operator()(uint32_t v, double sum) const {
    const double val = (v == seed ? tele : 0.0) + d * sum;
    x[v] = val;
    const uint32_t od = outdeg[v];
    cnext[v] = od ? val / (double)od : 0.0;
  }
};

__global__ void k_ppr1_init(uint64_t n, uint32_t seed, const uint32_t* __restrict__ outdeg, double tele, double* __restrict__ x,
                            double* __restrict__ c0, double* __restrict__ c1) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const double t = (v == seed) ? tele : 0.0;
    const uint32_t od = outdeg[v];
    const double c = od ? t / (double)od : 0.0;
    x[v] = t;
    c0[v] = c;
    c1[v] = c;
  }
}

// ---------------------------------------------------------------------------------------------
// weighted PageRank and its adjoint
// ---------------------------------------------------------------------------------------------
struct GatherWeighted {  // sum_a p[a] * x[col[a]]
  const uint32_t* __restrict__ col;
  const double* __restrict__ p;
  const double* __restrict__ x;
  __device__ __forceinline__ double operator()(uint32_t, uint64_t a) const { return __ldg(p + a) * x[__ldg(col + a)]; }
};
struct GatherW {  // sum_a w[a]
  const double* __restrict__ w;
  __device__ __forceinline__ double operator()(uint32_t, uint64_t a) const { return __ldg(w + a); }
};
struct FinishStore {
  double* __restrict__ out;
  __device__ __forceinline__ void operator()(uint32_t v, double s) const { out[v] = s; }
};

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double val) {
  // non-negative doubles order like their bit patterns
  atomicMax((unsigned long long*)addr, (unsigned long long)__double_as_longlong(val));
}

// y[v] = base[v] + d*sum (base = (1-d)*pers for the forward, c for the adjoint); tracks max|dy|
struct FinishAffine {
  double* __restrict__ y;
  const double* __restrict__ xprev;
  const double* __restrict__ base;  // null: constant base_c
  double base_c, scale, d;
  double* __restrict__ maxdiff;
  __device__ __forceinline__ void operator()(uint32_t v, double sum) const {
    const double b = base ? scale * base[v] : base_c;
    const double val = b + d * sum;
    y[v] = val;
    atomic_max_nonneg(maxdiff, fabs(val - xprev[v]));
  }
};

__global__ void k_affine_init(uint64_t n, const double* __restrict__ base, double base_c, double scale, double* __restrict__ a,
                              double* __restrict__ b) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const double x = base ? scale * base[v] : base_c;
    a[v] = x;
    b[v] = x;
  }
}

// p[a] = w[a] / s[row(a)] over the CSR, and pw[slot] = rw[slot] / s[rcol[slot]] over the CSC
struct VisitNormalise {
  const double* __restrict__ w;
  const double* __restrict__ s;
  double* __restrict__ p;
};

__global__ void k_csc_normalise(uint64_t m, const uint32_t* __restrict__ rcol, const double* __restrict__ rw,
                                const double* __restrict__ s, double* __restrict__ pw) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < m; a += (uint64_t)gridDim.x * blockDim.x)
    pw[a] = rw[a] / s[rcol[a]];
}
__global__ void k_csr_normalise(uint64_t n, const uint64_t* __restrict__ off, const double* __restrict__ w,
                                const double* __restrict__ s, double* __restrict__ p) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t u = warp; u < n; u += nwarps) {
    const double su = s[u];
    for (uint64_t a = off[u] + lane; a < off[u + 1]; a += 32) p[a] = w[a] / su;
  }
}

// grad_w[a] = d * r[u] / s[u] * (lambda[col[a]] - pl[u]) for every arc of row u
__global__ void k_grad_w(uint64_t n, const uint64_t* __restrict__ off, const uint32_t* __restrict__ col, const double* __restrict__ r,
                         const double* __restrict__ s, const double* __restrict__ lambda, const double* __restrict__ pl, double d,
                         double* __restrict__ gw) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t u = warp; u < n; u += nwarps) {
    const uint64_t a0 = off[u], a1 = off[u + 1];
    if (a0 == a1) continue;
    const double f = d * r[u] / s[u];
    const double plu = pl[u];
    for (uint64_t a = a0 + lane; a < a1; a += 32) gw[a] = f * (lambda[col[a]] - plu);
  }
}

__global__ void k_scale(uint64_t n, const double* __restrict__ x, double f, double* __restrict__ y) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) y[v] = f * x[v];
}

// Row sums s, CSR-normalised p and CSC-normalised pw of the FP64 weights (kept in workspace).
struct WeightedPrep {
  double* s;
  double* p;
  double* pw;
};
static int weighted_prep(gre_graph g, WeightedPrep* wp) {
  if (!g->w64 || !g->rw64) {
    set_error("weighted PageRank needs FP64 arc weights (gre_graph_set_weights_f64)");
    return GRE_INVALID_ARG;
  }
  GRE_CHECK(ensure_bins(g, false));
  GRE_CHECK(ws_array(g, WS_I, g->n, &wp->s));
  GRE_CHECK(ws_array(g, WS_J, g->m, &wp->p));
  GRE_CHECK(ws_array(g, WS_K, g->m, &wp->pw));
  double* partial;
  GRE_CHECK(ws_array(g, WS_H, g->bins_out.n_partials + 1, &partial));
  GRE_CUDA(cudaMemsetAsync(wp->s, 0, sizeof(double) * g->n, g->stream));
  GRE_CHECK(rows::reduce_rows(g->bins_out, g->off, GatherW{g->w64}, FinishStore{wp->s}, partial, g->stream));
  k_csr_normalise<<<grid_for(g->n * 32, 256), 256, 0, g->stream>>>(g->n, g->off, g->w64, wp->s, wp->p);
  k_csc_normalise<<<grid_for(g->m, 256), 256, 0, g->stream>>>(g->m, g->rcol, g->rw64, wp->s, wp->pw);
  GRE_LAUNCH_CHECK();
  return GRE_SUCCESS;
}

// Jacobi iteration y = base + d * (A x) with A given by (bins, off, col, p), to tolerance.
static int affine_solve(gre_graph g, const DegreeBins& B, const uint64_t* off, const uint32_t* col, const double* p,
                        const double* base, double scale, double base_c, double d, double tol, uint32_t max_iters,
                        double* xa, double* xb, double** result, uint32_t* iters_done, gre_stats* st) {
  double* partial;
  double* maxdiff;
  GRE_CHECK(ws_array(g, WS_H, B.n_partials + 1, &partial));
  GRE_CHECK(ws_array(g, WS_COUNTERS, 2, &maxdiff));
  k_affine_init<<<grid_for(g->n, 256), 256, 0, g->stream>>>(g->n, base, base_c, scale, xa, xb);
  // one iteration x -> y; maxdiff holds that iteration's largest change (reset first)
  auto iteration = [&](double* x, double* y) -> int {
    GRE_CUDA(cudaMemsetAsync(maxdiff, 0, sizeof(double), g->stream));
    // rows without arcs keep base (set by init in both buffers)
    return rows::reduce_rows(B, off, GatherWeighted{col, p, x}, FinishAffine{y, x, base, base_c, scale, d, maxdiff}, partial,
                             g->stream);
  };
  // convergence is read every check_every iterations (an even number: the buffers are back in
  // place), so that block is recorded once as a CUDA graph and replayed until it converges
  const uint32_t check_every = 4;
  Recorded rec;
  GRE_CHECK(rec.record(g->stream, [&]() {
    int e = 0;
    for (uint32_t i = 0; i < check_every && !e; ++i) e = (i & 1) ? iteration(xb, xa) : iteration(xa, xb);
    return e;
  }));
  double* x = xa;
  double* y = xb;
  uint32_t it = 0;
  while (it < max_iters) {
    if (it + check_every <= max_iters && x == xa) {
      GRE_CHECK(rec.replay(g->stream));
      it += check_every;
    } else {
      GRE_CHECK(iteration(x, y));
      std::swap(x, y);
      ++it;
    }
    if (it % check_every == 0 || it == max_iters) {
      double h = 0;
      GRE_CUDA(cudaMemcpyAsync(&h, maxdiff, sizeof h, cudaMemcpyDeviceToHost, g->stream));
      GRE_CUDA(cudaStreamSynchronize(g->stream));
      if (h <= tol) break;
    }
  }
  *result = x;
  *iters_done = it;
  return GRE_SUCCESS;
}

}  // namespace gre

using namespace gre;

extern "C" {

int gre_pagerank(gre_graph g, int variant, double d, uint32_t iters, double* pr, gre_stats* st) {
  if (!g || !pr) return GRE_NULL;
  if ((variant != GRE_PR_REFERENCE && variant != GRE_PR_ITER) || !(d >= 0.0 && d < 1.0)) return GRE_INVALID_ARG;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  GRE_CHECK(ensure_bins(g, true));
  const uint64_t n = g->n;
  double *dout, *dpr, *c0, *c1, *partial;
  GRE_CHECK(prepare_output(g, pr, n, WS_OUTBUF, &dout));
  GRE_CHECK(perm_out_begin(g, dout, 1, 8, (void**)&dpr));
  GRE_CHECK(ws_array(g, WS_A, n, &c0));
  GRE_CHECK(ws_array(g, WS_B, n, &c1));
  GRE_CHECK(ws_array(g, WS_C, g->bins_in.n_partials + 1, &partial));
  const double tele = 1.0 - d;
  const bool refresh = variant == GRE_PR_ITER;
  RunTimer timer(g);
  k_pr_init<<<grid_for(n, 256), 256, 0, g->stream>>>(n, g->outdeg, tele, dpr, c0, refresh ? c1 : nullptr);
  GRE_LAUNCH_CHECK();
  // one superstep reads contributions `a` and (power iteration) writes the next ones to `b`
  auto superstep = [&](double* a, double* b) -> int {
    FinishPR fin{dpr, refresh ? b : nullptr, g->outdeg, tele, d};
    return rows::reduce_rows(g->bins_in, g->roff, GatherContrib{g->rcol, a}, fin, partial, g->stream);
  };
  // supersteps repeat with period 2 (the contribution buffers swap), 1 for the reference
  // variant: that period is recorded once as a CUDA graph and replayed
  const uint32_t period = refresh ? 2 : 1;
  uint32_t done = 0;
  if (iters >= 2 * period) {
    Recorded rec;
    GRE_CHECK(rec.record(g->stream, [&]() {
      int e = superstep(c0, c1);
      if (!e && refresh) e = superstep(c1, c0);
      return e;
    }));
    for (; done + period <= iters; done += period) GRE_CHECK(rec.replay(g->stream));
  }
  for (double *cur = c0, *nxt = c1; done < iters; ++done) {
    GRE_CHECK(superstep(cur, nxt));
    if (refresh) std::swap(cur, nxt);
  }
  GRE_CHECK(perm_out_end(g, dpr, dout, 1, 8));
  GRE_CHECK(finish_output(g, pr, dout, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = iters;
    for (uint32_t i = 0; i < iters; ++i) stats_record(st, rows::nonempty_rows(g->bins_in));
    st->arcs_traversed = g->m * (uint64_t)iters;
    st->traversed_edges = g->m * (uint64_t)iters;
    st->algo_bytes = pr_bytes_per_iter(n, g->m) * iters;
  }
  return GRE_SUCCESS;
}

int gre_ppr(gre_graph g, const uint32_t* seeds, uint32_t k, double d, uint32_t iters, int batched, double* out, gre_stats* st) {
  if (!g || !out || (k && !seeds)) return GRE_NULL;
  if (!(d >= 0.0 && d < 1.0)) return GRE_INVALID_ARG;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  if (k == 0) return GRE_SUCCESS;
  const uint64_t n = g->n;
  std::vector<uint32_t> hs(k);
  GRE_CUDA(cudaMemcpy(hs.data(), seeds, sizeof(uint32_t) * k, cudaMemcpyDefault));
  GRE_CHECK(map_ids(g, &hs, "gre_ppr"));
  GRE_CHECK(ensure_bins(g, true));
  const double tele = 1.0 - d;
  double *dfinal, *dout;
  GRE_CHECK(prepare_output(g, out, (uint64_t)k * n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, k, 8, (void**)&dout));
  RunTimer timer(g);
  if (!batched) {
    double *c0, *c1, *partial;
    GRE_CHECK(ws_array(g, WS_A, n, &c0));
    GRE_CHECK(ws_array(g, WS_B, n, &c1));
    GRE_CHECK(ws_array(g, WS_C, g->bins_in.n_partials + 1, &partial));
    for (uint32_t j = 0; j < k; ++j) {
      double* x = dout + (uint64_t)j * n;
      k_ppr1_init<<<grid_for(n, 256), 256, 0, g->stream>>>(n, hs[j], g->outdeg, tele, x, c0, c1);
      double* cur = c0;
      double* nxt = c1;
      for (uint32_t it = 0; it < iters; ++it) {
        GRE_CHECK(rows::reduce_rows(g->bins_in, g->roff, GatherContrib{g->rcol, cur}, FinishPPR1{x, nxt, g->outdeg, hs[j], tele, d},
                                    partial, g->stream));
        std::swap(cur, nxt);
      }
    }
    if (st) st->algo_bytes = (uint64_t)k * iters * pr_bytes_per_iter(n, g->m);
  } else {
    PprChunks pc;
    GRE_CHECK(ppr_chunks(g, &pc));
    double *x, *c0, *c1, *partial;
    uint32_t* dseeds;
    GRE_CHECK(ws_array(g, WS_A, n * kCols, &x));
    GRE_CHECK(ws_array(g, WS_B, n * kCols, &c0));
    GRE_CHECK(ws_array(g, WS_C, n * kCols, &c1));
    GRE_CHECK(ws_array(g, WS_D, (pc.nchunks + 1) * kCols, &partial));
    GRE_CHECK(ws_array(g, WS_E, kCols, &dseeds));
    const DegreeBins& B = g->bins_in;
    uint64_t short_rows = 0;
    for (int b = 0; b < 6; ++b) short_rows += B.count[b];  // rows longer than kPprChunk are skipped
    std::unique_ptr<Recorded> rec;
    uint32_t rec_kk = 0;
    for (uint32_t j0 = 0; j0 < k; j0 += kCols) {
      const uint32_t kk = (k - j0) < (uint32_t)kCols ? (k - j0) : (uint32_t)kCols;
      GRE_CUDA(cudaMemcpyAsync(dseeds, hs.data() + j0, sizeof(uint32_t) * kk, cudaMemcpyHostToDevice, g->stream));
      k_ppr_init<<<grid_for(n * kCols, 256), 256, 0, g->stream>>>(n, kk, dseeds, g->outdeg, tele, x, c0, c1);
      k_ppr_seed<<<1, 128, 0, g->stream>>>(kk, dseeds, g->outdeg, tele, x, c0, c1);
      auto superstep = [&](double* a, double* b) -> int {
        PprRow R{g->roff, g->rcol, a};
        PprFinish F{x, b, g->outdeg, dseeds, kk, tele, d};
        if (short_rows) k_ppr_rows<<<grid_for(short_rows * 32, 256, 8), 256, 0, g->stream>>>(B.rows, short_rows, R, F);
        if (pc.nrows) {
          k_ppr_chunks<<<grid_for(pc.nchunks * 32, 256, 8), 256, 0, g->stream>>>(pc.rows, pc.row, pc.begin, pc.nchunks, R, partial);
          k_ppr_chunk_finish<<<grid_for(pc.nrows * 32, 256, 8), 256, 0, g->stream>>>(pc.rows, pc.nrows, pc.first, partial, F);
        }
        GRE_LAUNCH_CHECK();
        return GRE_SUCCESS;
      };
      // two supersteps (the buffers swap back) recorded once per block width, then replayed
      if (!rec || rec_kk != kk) {
        rec.reset(new Recorded());
        rec_kk = kk;
        GRE_CHECK(rec->record(g->stream, [&]() {
          int e = superstep(c0, c1);
          if (!e) e = superstep(c1, c0);
          return e;
        }));
      }
      uint32_t it = 0;
      for (; it + 2 <= iters; it += 2) GRE_CHECK(rec->replay(g->stream));
      if (it < iters) GRE_CHECK(superstep(c0, c1));
      k_ppr_transpose<<<grid_for((uint64_t)kk * n, 256), 256, 0, g->stream>>>(n, kk, x, dout + (uint64_t)j0 * n);
      GRE_LAUNCH_CHECK();
    }
    if (st) {
      const uint64_t passes = (k + kCols - 1) / kCols;
      st->algo_bytes = passes * iters * (8 * (n + 1) + 4 * g->m + (uint64_t)kCols * (8 * g->m + 24 * n));
    }
  }
  GRE_CHECK(perm_out_end(g, dout, dfinal, k, 8));
  GRE_CHECK(finish_output(g, out, dfinal, (uint64_t)k * n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = iters;
    st->arcs_traversed = g->m * (uint64_t)iters * k;
    st->traversed_edges = st->arcs_traversed;
  }
  return GRE_SUCCESS;
}

int gre_pagerank_weighted(gre_graph g, double d, const double* pers, double tol, uint32_t max_iters, double* r, gre_stats* st) {
  if (!g || !r) return GRE_NULL;
  if (!(d >= 0.0 && d < 1.0) || !(tol >= 0.0)) return GRE_INVALID_ARG;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  GRE_CHECK(ensure_bins(g, true));
  WeightedPrep wp;
  GRE_CHECK(weighted_prep(g, &wp));
  const double* dpers;
  double *dr, *xa, *xb, *res;
  GRE_CHECK(stage_input(g, pers, n, WS_G, &dpers));
  GRE_CHECK(perm_in(g, dpers, 8, WS_PERM_IN, (const void**)&dpers));
  GRE_CHECK(prepare_output(g, r, n, WS_OUTBUF, &dr));
  GRE_CHECK(ws_array(g, WS_A, n, &xa));
  GRE_CHECK(ws_array(g, WS_B, n, &xb));
  RunTimer timer(g);
  uint32_t done = 0;
  GRE_CHECK(affine_solve(g, g->bins_in, g->roff, g->rcol, wp.pw, dpers, 1.0 - d, 1.0 - d, d, tol, max_iters, xa, xb, &res, &done, st));
  if (g->perm) GRE_CHECK(perm_out_end(g, res, dr, 1, 8));
  else GRE_CUDA(cudaMemcpyAsync(dr, res, sizeof(double) * n, cudaMemcpyDeviceToDevice, g->stream));
  GRE_CHECK(finish_output(g, r, dr, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = done;
    st->arcs_traversed = g->m * (uint64_t)done;
    st->traversed_edges = st->arcs_traversed;
    st->algo_bytes = (uint64_t)done * (8 * (n + 1) + 20 * g->m + 16 * n);
  }
  return done < max_iters || max_iters == 0 ? GRE_SUCCESS : GRE_UNFINISHED;
}

int gre_pagerank_adjoint(gre_graph g, double d, const double* r, const double* c, double tol, uint32_t max_iters, double* lambda,
                         double* grad_pers, double* grad_w, gre_stats* st) {
  if (!g || !r || !c || !grad_w) return GRE_NULL;
  if (!(d > 0.0 && d < 1.0) || !(tol >= 0.0)) return GRE_INVALID_ARG;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n, m = g->m;
  GRE_CHECK(ensure_bins(g, true));
  WeightedPrep wp;
  GRE_CHECK(weighted_prep(g, &wp));
  const double *dr, *dc;
  double *xa, *xb, *res, *pl, *dgw, *dlam = nullptr, *dgp = nullptr;
  GRE_CHECK(stage_input(g, r, n, WS_F, &dr));
  GRE_CHECK(stage_input(g, c, n, WS_G, &dc));
  GRE_CHECK(perm_in(g, dr, 8, WS_PERM_IN, (const void**)&dr));
  GRE_CHECK(perm_in(g, dc, 8, WS_PERM_IN2, (const void**)&dc));
  GRE_CHECK(ws_array(g, WS_A, n, &xa));
  GRE_CHECK(ws_array(g, WS_B, n, &xb));
  GRE_CHECK(ws_array(g, WS_C, n, &pl));
  double* dgw_final;
  GRE_CHECK(prepare_output(g, grad_w, m, WS_OUTBUF, &dgw_final));
  dgw = dgw_final;
  if (g->perm) GRE_CHECK(ws_array(g, WS_PERM_OUT, m, &dgw));  // internal arc order first
  if (lambda) GRE_CHECK(prepare_output(g, lambda, n, WS_D, &dlam));
  if (grad_pers) GRE_CHECK(prepare_output(g, grad_pers, n, WS_E, &dgp));
  RunTimer timer(g);
  uint32_t done = 0;
  // lambda = c + d P lambda: pull over the CSR rows (out-arcs) with p = W/s
  GRE_CHECK(affine_solve(g, g->bins_out, g->off, g->col, wp.p, dc, 1.0, 0.0, d, tol, max_iters, xa, xb, &res, &done, st));
  // pl[u] = sum_k P_uk lambda_k (rows without arcs keep 0)
  double* partial;
  GRE_CHECK(ws_array(g, WS_H, g->bins_out.n_partials + 1, &partial));
  GRE_CUDA(cudaMemsetAsync(pl, 0, sizeof(double) * n, g->stream));
  GRE_CHECK(rows::reduce_rows(g->bins_out, g->off, GatherWeighted{g->col, wp.p, res}, FinishStore{pl}, partial, g->stream));
  k_grad_w<<<grid_for(n * 32, 256), 256, 0, g->stream>>>(n, g->off, g->col, dr, wp.s, res, pl, d, dgw);
  GRE_LAUNCH_CHECK();
  if (g->perm) GRE_CHECK(arcs_to_caller(g, dgw, dgw_final, 8));
  dgw = dgw_final;
  if (dgp) {
    // (1-d) lambda into pl (free now), then to caller order
    k_scale<<<grid_for(n, 256), 256, 0, g->stream>>>(n, res, 1.0 - d, g->perm ? pl : dgp);
    if (g->perm) GRE_CHECK(perm_out_end(g, pl, dgp, 1, 8));
  }
  if (dlam) {
    if (g->perm) GRE_CHECK(perm_out_end(g, res, dlam, 1, 8));
    else GRE_CUDA(cudaMemcpyAsync(dlam, res, sizeof(double) * n, cudaMemcpyDeviceToDevice, g->stream));
  }
  GRE_LAUNCH_CHECK();
  GRE_CHECK(finish_output(g, grad_w, dgw, m));
  if (lambda) GRE_CHECK(finish_output(g, lambda, dlam, n));
  if (grad_pers) GRE_CHECK(finish_output(g, grad_pers, dgp, n));
  GRE_CHECK(timer.stop(st));
  if (st) {
    st->supersteps = done;
    st->arcs_traversed = m * (uint64_t)(done + 2);
    st->traversed_edges = st->arcs_traversed;
    st->algo_bytes = (uint64_t)(done + 1) * (8 * (n + 1) + 20 * m + 16 * n) + (8 * (n + 1) + 4 * m + 8 * m + 8 * m + 24 * n);
  }
  return done < max_iters || max_iters == 0 ? GRE_SUCCESS : GRE_UNFINISHED;
}

}  // extern "C"
