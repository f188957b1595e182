// C ABI of the reference-semantics engine: the reference plugins (plugins.cuh) on the device
// SynchronousEngine (gre/vertex_code.cuh), driven like the reference drivers usr/test_*.cpp.
#include "gre_internal.cuh"
#include "plugins.cuh"

namespace gre {

static DeviceGraphView view_of(gre_graph g) { return DeviceGraphView{g->n, g->off, g->col, g->roff, g->rcol, g->rarc}; }

template <class VC>
static int run_engine(gre_graph g, VC& vc, int dir, const SourceSet& src, uint32_t max_ss, void* scratch,
                      gre_stats* st, long* supersteps, uint64_t* last_active) {
  SynchronousEngine<VC> eng(view_of(g), vc, g->stream, scratch);
  eng.configMaxSupersteps(max_ss);
  eng.dir_for_arcs_ = dir;
  const int sms = num_sms();
  cudaError_t e;
  if (dir == GRE_DIR_OUT) e = eng.template run<VC_OUT>(src, sms);
  else if (dir == GRE_DIR_IN) e = eng.template run<VC_IN>(src, sms);
  else e = eng.template run<VC_INOUT>(src, sms);
  if (e != cudaSuccess) return cuda_status(e, "SynchronousEngine::run", __FILE__, __LINE__);
  if (st) {
    st->supersteps += (uint32_t)eng.getSuperstepCount();
    for (uint64_t a : eng.activeCounts()) stats_record(st, a);
    st->arcs_traversed += eng.arcsScanned();
  }
  if (supersteps) *supersteps = eng.getSuperstepCount();
  if (last_active) *last_active = eng.activeCounts().empty() ? 0 : eng.activeCounts().back();
  return GRE_SUCCESS;
}

template <class T>
static int ws_array(gre_graph g, int slot, uint64_t count, T** p) {
  void* v = nullptr;
  GRE_CHECK(g->ws.get(slot, sizeof(T) * (count ? count : 1), &v));
  *p = (T*)v;
  return GRE_SUCCESS;
}

__global__ void k_bc_accumulate(uint64_t n, uint32_t s, const double* __restrict__ dep, double* __restrict__ bc) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    if (v != s) bc[v] += dep[v];
}

}  // namespace gre

using namespace gre;

extern "C" {

int gre_vc_pagerank(gre_graph g, int variant, uint32_t max_supersteps, double* pr, gre_stats* st) {
  if (!g || !pr) return GRE_NULL;
  if (variant != GRE_PR_REFERENCE && variant != GRE_PR_ITER) return GRE_INVALID_ARG;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  double *dfinal, *dpr, *scat, *comb;
  void* scratch;
  GRE_CHECK(prepare_output(g, pr, n, WS_OUTBUF, &dfinal));
  GRE_CHECK(perm_out_begin(g, dfinal, 1, 8, (void**)&dpr));
  GRE_CHECK(ws_array(g, WS_B, n, &scat));
  GRE_CHECK(ws_array(g, WS_C, n, &comb));
  GRE_CHECK(g->ws.get(WS_D, vc_scratch_bytes(n), &scratch));
  RunTimer timer(g);
  GRE_CUDA(cudaMemsetAsync(comb, 0, sizeof(double) * n, g->stream));  // allocCombineData(pr_combine, 0.0)
  double* stat;
  GRE_CHECK(ws_array(g, WS_COUNTERS, plugin_stats::kBlocks + 8, &stat));
  VcPageRank vc{dpr, scat, comb, g->outdeg, 0.15, 1.0 - 0.15, variant == GRE_PR_ITER, stat, st ? &st->plugin_value : nullptr};
  SourceSet all;
  all.all = true;
  GRE_CHECK(run_engine(g, vc, GRE_DIR_OUT, all, max_supersteps, scratch, st, nullptr, nullptr));
  GRE_CHECK(perm_out_end(g, dpr, dfinal, 1, 8));
  GRE_CHECK(finish_output(g, pr, dfinal, n));
  GRE_CHECK(timer.stop(st));
  if (st) st->traversed_edges = st->arcs_traversed;
  return GRE_SUCCESS;
}

}  // extern "C"

// internal-order result -> caller output (device or host); `slot` stages host outputs
template <class T>
static int emit(gre_graph g, T* out, const T* internal, int slot) {
  if (!out) return GRE_SUCCESS;
  T* dout;
  GRE_CHECK(prepare_output(g, out, g->n, slot, &dout));
  if (g->perm) GRE_CHECK(perm_out_end(g, internal, dout, 1, sizeof(T)));
  else if (dout != internal) GRE_CUDA(cudaMemcpyAsync(dout, internal, sizeof(T) * g->n, cudaMemcpyDeviceToDevice, g->stream));
  return finish_output(g, out, dout, g->n);
}

extern "C" {

int gre_vc_bfs(gre_graph g, uint32_t src, int dir, uint64_t* pred, int32_t* level, gre_stats* st) {
  if (!g) return GRE_NULL;
  if (dir < GRE_DIR_OUT || dir > GRE_DIR_INOUT) return GRE_INVALID_ARG;
  GRE_CHECK(use_graph(g));
  std::vector<uint32_t> hs(1, src);
  GRE_CHECK(map_ids(g, &hs, "gre_vc_bfs"));
  stats_reset(st);
  const uint64_t n = g->n;
  unsigned long long *dpred, *scat, *comb;
  int32_t* dlevel;
  const uint32_t* dsrc;
  void* scratch;
  GRE_CHECK(ws_array(g, WS_A, n, &dpred));
  GRE_CHECK(ws_array(g, WS_I, n, &dlevel));
  GRE_CHECK(ws_array(g, WS_B, n, &scat));
  GRE_CHECK(ws_array(g, WS_C, n, &comb));
  GRE_CHECK(g->ws.get(WS_D, vc_scratch_bytes(n), &scratch));
  RunTimer timer(g);
  GRE_CHECK(stage_input(g, hs.data(), 1, WS_E, &dsrc));
  GRE_CUDA(cudaMemsetAsync(dpred, 0xff, sizeof(unsigned long long) * n, g->stream));  // allocVertexData(pred, -1)
  GRE_CUDA(cudaMemsetAsync(comb, 0xff, sizeof(unsigned long long) * n, g->stream));   // allocCombineData(pred_combine, -1)
  GRE_CUDA(cudaMemsetAsync(dlevel, 0xff, sizeof(int32_t) * n, g->stream));
  VcBFS vc{dpred, scat, comb, dlevel, g->perm, 0};
  SourceSet s;
  s.dev_vertices = dsrc;
  s.count = 1;
  GRE_CHECK(run_engine(g, vc, dir, s, 1024, scratch, st, nullptr, nullptr));
  GRE_CHECK(emit(g, (unsigned long long*)pred, dpred, WS_OUTBUF));
  GRE_CHECK(emit(g, level, dlevel, WS_OUTBUF2));
  GRE_CHECK(timer.stop(st));
  return GRE_SUCCESS;
}

int gre_vc_sssp(gre_graph g, uint32_t src, uint32_t max_supersteps, uint32_t* dist, gre_stats* st) {
  if (!g || !dist) return GRE_NULL;
  if (!g->w32) {
    set_error("gre_vc_sssp: the graph has no uint32 weights (gre_graph_set_weights_*)");
    return GRE_INVALID_ARG;
  }
  GRE_CHECK(use_graph(g));
  std::vector<uint32_t> hs(1, src);
  GRE_CHECK(map_ids(g, &hs, "gre_vc_sssp"));
  stats_reset(st);
  const uint64_t n = g->n;
  uint32_t *states, *last;
  const uint32_t* dsrc;
  void* scratch;
  GRE_CHECK(ws_array(g, WS_A, n, &states));
  GRE_CHECK(ws_array(g, WS_B, n, &last));
  GRE_CHECK(g->ws.get(WS_D, vc_scratch_bytes(n), &scratch));
  RunTimer timer(g);
  GRE_CHECK(stage_input(g, hs.data(), 1, WS_E, &dsrc));
  GRE_CUDA(cudaMemsetAsync(states, 0xff, sizeof(uint32_t) * n, g->stream));  // numeric_limits<dist_t>::max()
  GRE_CUDA(cudaMemsetAsync(last, 0, sizeof(uint32_t) * n, g->stream));
  VcSSSP vc{states, last, g->w32};
  SourceSet s;
  s.dev_vertices = dsrc;
  s.count = 1;
  uint64_t last_active = 0;
  GRE_CHECK(run_engine(g, vc, GRE_DIR_OUT, s, max_supersteps, scratch, st, nullptr, &last_active));
  GRE_CHECK(emit(g, dist, states, WS_OUTBUF));
  GRE_CHECK(timer.stop(st));
  return last_active ? GRE_UNFINISHED : GRE_SUCCESS;
}

int gre_vc_pagerank_delta(gre_graph g, uint32_t max_supersteps, double* pr, gre_stats* st) {
  if (!g || !pr) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  double *dpr, *scat, *comb;
  void* scratch;
  GRE_CHECK(ws_array(g, WS_A, n, &dpr));
  GRE_CHECK(ws_array(g, WS_B, n, &scat));
  GRE_CHECK(ws_array(g, WS_C, n, &comb));
  GRE_CHECK(g->ws.get(WS_D, vc_scratch_bytes(n), &scratch));
  RunTimer timer(g);
  GRE_CUDA(cudaMemsetAsync(comb, 0, sizeof(double) * n, g->stream));  // allocCombineData(pr_combine, 0.0)
  VcPageRankDelta vc{dpr, scat, comb, g->outdeg, 0.15, 1.0 - 0.15, 1e-5};
  SourceSet all;
  all.all = true;
  uint64_t last_active = 0;
  GRE_CHECK(run_engine(g, vc, GRE_DIR_OUT, all, max_supersteps, scratch, st, nullptr, &last_active));
  GRE_CHECK(emit(g, pr, dpr, WS_OUTBUF));
  GRE_CHECK(timer.stop(st));
  if (st) st->traversed_edges = st->arcs_traversed;
  return last_active ? GRE_UNFINISHED : GRE_SUCCESS;
}

__global__ void k_split_sssp1(uint64_t n, const unsigned long long* __restrict__ states, uint32_t* __restrict__ dist,
                              unsigned long long* __restrict__ pred) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long x = states[v];
    const uint32_t d = (uint32_t)(x >> 32);
    dist[v] = d;
    pred[v] = d == 0xffffffffu ? ~0ull : (x & 0xffffffffull);  // _Data(): pred -1 when unreached
  }
}

int gre_vc_sssp1(gre_graph g, uint32_t src, uint32_t max_supersteps, uint32_t* dist, uint64_t* pred, gre_stats* st) {
  if (!g || !dist || !pred) return GRE_NULL;
  if (!g->w32) {
    set_error("gre_vc_sssp1: the graph has no uint32 weights (gre_graph_set_weights_*)");
    return GRE_INVALID_ARG;
  }
  GRE_CHECK(use_graph(g));
  std::vector<uint32_t> hs(1, src);
  GRE_CHECK(map_ids(g, &hs, "gre_vc_sssp1"));
  stats_reset(st);
  const uint64_t n = g->n;
  unsigned long long *states, *dpred;
  uint32_t *last, *ddist;
  const uint32_t* dsrc;
  void* scratch;
  GRE_CHECK(ws_array(g, WS_A, n, &states));
  GRE_CHECK(ws_array(g, WS_B, n, &last));
  GRE_CHECK(ws_array(g, WS_C, n, &ddist));
  GRE_CHECK(ws_array(g, WS_F, n, &dpred));
  GRE_CHECK(g->ws.get(WS_D, vc_scratch_bytes(n), &scratch));
  RunTimer timer(g);
  GRE_CHECK(stage_input(g, hs.data(), 1, WS_E, &dsrc));
  GRE_CUDA(cudaMemsetAsync(states, 0xff, sizeof(unsigned long long) * n, g->stream));  // _Data(): dist max, pred -1
  GRE_CUDA(cudaMemsetAsync(last, 0xff, sizeof(uint32_t) * n, g->stream));
  VcSSSP1 vc{states, last, g->w32, g->perm};
  SourceSet s;
  s.dev_vertices = dsrc;
  s.count = 1;
  uint64_t last_active = 0;
  GRE_CHECK(run_engine(g, vc, GRE_DIR_OUT, s, max_supersteps, scratch, st, nullptr, &last_active));
  k_split_sssp1<<<grid_for(n, 256), 256, 0, g->stream>>>(n, states, ddist, dpred);
  GRE_LAUNCH_CHECK();
  GRE_CHECK(emit(g, dist, ddist, WS_OUTBUF));
  GRE_CHECK(emit(g, (unsigned long long*)pred, dpred, WS_OUTBUF2));
  GRE_CHECK(timer.stop(st));
  return last_active ? GRE_UNFINISHED : GRE_SUCCESS;
}

int gre_vc_count_in(gre_graph g, int dir, uint32_t max_supersteps, int32_t* count, gre_stats* st) {
  if (!g || !count) return GRE_NULL;
  if (dir < GRE_DIR_OUT || dir > GRE_DIR_INOUT) return GRE_INVALID_ARG;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  int32_t *cn, *scat, *comb;
  void* scratch;
  GRE_CHECK(ws_array(g, WS_A, n, &cn));
  GRE_CHECK(ws_array(g, WS_B, n, &scat));
  GRE_CHECK(ws_array(g, WS_C, n, &comb));
  GRE_CHECK(g->ws.get(WS_D, vc_scratch_bytes(n), &scratch));
  RunTimer timer(g);
  GRE_CUDA(cudaMemsetAsync(cn, 0, sizeof(int32_t) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(comb, 0, sizeof(int32_t) * n, g->stream));  // allocCombineData(cn_combine, 0)
  double* stat;
  GRE_CHECK(ws_array(g, WS_COUNTERS, 8, &stat));
  VcCountIn vc{cn, scat, comb, stat, st ? &st->plugin_count : nullptr};
  SourceSet all;
  all.all = true;
  GRE_CHECK(run_engine(g, vc, dir, all, max_supersteps, scratch, st, nullptr, nullptr));
  GRE_CHECK(emit(g, count, cn, WS_OUTBUF));
  GRE_CHECK(timer.stop(st));
  return GRE_SUCCESS;
}

int gre_vc_cc(gre_graph g, uint32_t* label, gre_stats* st) {
  if (!g || !label) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  uint32_t *cc, *scat, *comb;
  void* scratch;
  GRE_CHECK(ws_array(g, WS_A, n, &cc));
  GRE_CHECK(ws_array(g, WS_B, n, &scat));
  GRE_CHECK(ws_array(g, WS_C, n, &comb));
  GRE_CHECK(g->ws.get(WS_D, vc_scratch_bytes(n), &scratch));
  RunTimer timer(g);
  GRE_CUDA(cudaMemsetAsync(cc, 0xff, sizeof(uint32_t) * n, g->stream));
  GRE_CUDA(cudaMemsetAsync(comb, 0xff, sizeof(uint32_t) * n, g->stream));
  double* stat;
  GRE_CHECK(ws_array(g, WS_COUNTERS, 8, &stat));
  VcCC vc{cc, scat, comb, g->perm, stat, st ? &st->plugin_count : nullptr};
  SourceSet all;
  all.all = true;
  GRE_CHECK(run_engine(g, vc, GRE_DIR_INOUT, all, 1024, scratch, st, nullptr, nullptr));
  GRE_CHECK(emit(g, label, cc, WS_OUTBUF));
  GRE_CHECK(timer.stop(st));
  return GRE_SUCCESS;
}

int gre_vc_bc(gre_graph g, const uint32_t* srcs, uint32_t nsrc, double* bc, gre_stats* st) {
  if (!g || !bc || (nsrc && !srcs)) return GRE_NULL;
  GRE_CHECK(use_graph(g));
  stats_reset(st);
  const uint64_t n = g->n;
  std::vector<uint32_t> hs(nsrc);
  if (nsrc) GRE_CUDA(cudaMemcpy(hs.data(), srcs, sizeof(uint32_t) * nsrc, cudaMemcpyDefault));
  GRE_CHECK(map_ids(g, &hs, "gre_vc_bc"));
  int32_t* level;
  double *sigma, *fscat, *fsum, *dep, *pathwgt, *bsum, *dbc;
  uint32_t* dsrc;
  void* scratch;
  GRE_CHECK(ws_array(g, WS_J, n, &dbc));
  GRE_CHECK(ws_array(g, WS_A, n, &level));
  GRE_CHECK(ws_array(g, WS_B, n, &sigma));
  GRE_CHECK(ws_array(g, WS_C, n, &fscat));
  GRE_CHECK(ws_array(g, WS_F, n, &fsum));
  GRE_CHECK(ws_array(g, WS_G, n, &dep));
  GRE_CHECK(ws_array(g, WS_H, n, &pathwgt));
  GRE_CHECK(ws_array(g, WS_I, n, &bsum));
  GRE_CHECK(ws_array(g, WS_E, 1, &dsrc));
  GRE_CHECK(g->ws.get(WS_D, vc_scratch_bytes(n), &scratch));
  RunTimer timer(g);
  GRE_CUDA(cudaMemsetAsync(dbc, 0, sizeof(double) * n, g->stream));
  for (uint32_t s : hs) {
    GRE_CUDA(cudaMemcpyAsync(dsrc, &s, sizeof s, cudaMemcpyHostToDevice, g->stream));
    // Forward: vtxData() = {level -1, numPaths 0}; scatter/combine arrays start at 0
    GRE_CUDA(cudaMemsetAsync(level, 0xff, sizeof(int32_t) * n, g->stream));
    GRE_CUDA(cudaMemsetAsync(sigma, 0, sizeof(double) * n, g->stream));
    GRE_CUDA(cudaMemsetAsync(fscat, 0, sizeof(double) * n, g->stream));
    GRE_CUDA(cudaMemsetAsync(fsum, 0, sizeof(double) * n, g->stream));
    VcForward fw{level, sigma, fscat, fsum, 1};
    SourceSet one;
    one.dev_vertices = dsrc;
    one.count = 1;
    GRE_CHECK(run_engine(g, fw, GRE_DIR_OUT, one, 1024, scratch, st, nullptr, nullptr));
    const int nLevels = fw.currLevel;  // usr/test_bc.cpp:86
    GRE_CUDA(cudaMemsetAsync(dep, 0, sizeof(double) * n, g->stream));
    GRE_CUDA(cudaMemsetAsync(pathwgt, 0, sizeof(double) * n, g->stream));
    GRE_CUDA(cudaMemsetAsync(bsum, 0, sizeof(double) * n, g->stream));
    VcBackward bw{level, sigma, dep, pathwgt, bsum, 0};
    SourceSet all;
    all.all = true;
    for (int i = nLevels - 2; i >= 0; --i) {  // usr/test_bc.cpp:99-105
      bw.currLevel = i;
      GRE_CHECK(run_engine(g, bw, GRE_DIR_IN, all, 1024, scratch, st, nullptr, nullptr));
    }
    k_bc_accumulate<<<grid_for(n, 256), 256, 0, g->stream>>>(n, s, dep, dbc);
    GRE_LAUNCH_CHECK();
  }
  GRE_CHECK(emit(g, bc, dbc, WS_OUTBUF));
  GRE_CHECK(timer.stop(st));
  return GRE_SUCCESS;
}

}  // extern "C"
