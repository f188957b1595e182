/*
 * gre_gpu.h — C ABI of the B200-native GRE superstep engine (libgre_gpu.so).
 *
 * This is the drop-in boundary for the hot path of the reference GRE engine
 * (NCIC-PARALLEL/Graphine): the vertex-centric superstep init -> scatter -> combine -> apply ->
 * vote-to-halt of SynchronousEngine (include/Engine/Engine.hpp:180-406,437-798) for the
 * PageRank, BFS, SSSP, ConnectedComponents and BC plugins (include/Kernels/), together
 * with the `<prefix>.meta` + `<prefix>.edges.<i>` loader (include/Graph/GraphIngress.hpp).
 * The reference is a header-only C++ template library with no FFI; each entry point below
 * names the reference function or driver step whose role it takes.
 *
 * Conventions
 *  - Every call returns a status code (gre_status below) and never exits the process.
 *  - Vertex ids are uint32, arc offsets uint64 (the reference: lvid_t = uint32,
 *    lidx_t = size_t; include/Types.hpp:13-18).
 *  - Buffers passed in or out may live in host memory or in device memory of the graph's
 *    device; the library checks which with cudaPointerGetAttributes and copies as needed.
 *    Outputs are caller-allocated.  Host outputs are complete when the call returns.
 *  - One CUDA stream per graph handle.  Calls on one handle are serialised by the caller;
 *    distinct handles may be used from different threads.  Each call first orders the graph's
 *    stream after the work issued so far on the legacy default stream (where PyTorch's default
 *    stream and stream-less kernels and copies run), so device buffers written or still read
 *    there are safe to pass; work on other streams of the caller must be complete (synchronise
 *    it) before a call that reads or writes its buffers, and during a stream capture the caller
 *    orders its buffers itself.  Device outputs, like host outputs, are complete on return.
 *  - Symbols under "host utilities" run on the CPU only and need no GPU.
 */
#ifndef GRE_GPU_H
#define GRE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes 0..8 keep the values of enum GRE_Status (include/Status.hpp:5-14). */
enum gre_status {
  GRE_SUCCESS = 0,
  GRE_FAILURE = 1,
  GRE_NOBUFFER = 2,
  GRE_NULL = 3,
  GRE_FINISHED = 4,
  GRE_UNFINISHED = 5, /* also: max supersteps reached before the frontier emptied */
  GRE_INITIALIZED = 6,
  GRE_UNINITIALIZED = 7,
  GRE_NOT_IMPLEMENTED = 8,
  GRE_INVALID_ARG = 9, /* added: bad size, vertex id out of range, missing weights ... */
  GRE_IO_ERROR = 10,   /* added: missing/garbled .meta / .edges.<i> / .roots */
  GRE_CUDA_ERROR = 11, /* added: a CUDA runtime call failed (see gre_last_error) */
  GRE_OOM = 12,        /* added: device or host allocation failed */
  GRE_TIMEOUT = 13,    /* added: a bounded device-side wait gave up */
  GRE_NO_DEVICE = 14   /* added: no usable CUDA device */
};

/* Edge directions: enum Dir {Out, In, InOut} (include/Types.hpp:33). */
enum gre_dir { GRE_DIR_OUT = 0, GRE_DIR_IN = 1, GRE_DIR_INOUT = 2 };

/* Graph flags for the loaders (OR-ed with a direction). */
enum gre_graph_flags {
  GRE_GRAPH_SYMMETRIC = 0x10, /* every arc (u,v) has its reverse: the CSR doubles as CSC */
  GRE_GRAPH_REORDER = 0x20    /* store vertices by decreasing degree (gre_graph_reorder) */
};

/* PageRank variants. */
enum gre_pr_variant {
  GRE_PR_REFERENCE = 0, /* Kernels/PageRank.hpp verbatim: pr_scatter never refreshed */
  GRE_PR_ITER = 1       /* power iteration: pr_scatter = pr/outdeg refreshed in apply */
};

#define GRE_MAX_RECORDED_SUPERSTEPS 1024 /* default max_nSupersteps (Engine.hpp:108) */

/* Per-run statistics.  `active` mirrors the per-superstep line the reference prints
 * ("Superstep-k: Number of active vertices...", Engine.hpp:392-398). */
typedef struct gre_stats {
  uint32_t supersteps;     /* SynchronousEngine::getSuperstepCount() (Engine.hpp:1307-1309) */
  uint32_t n_recorded;     /* valid entries of active[] */
  uint64_t arcs_traversed; /* arcs the kernels scanned */
  uint64_t traversed_edges;/* edges counted for TEPS (definition per algorithm) */
  uint64_t algo_bytes;     /* algorithmic HBM bytes of the run (byte model of each kernel) */
  double device_ms;        /* device time of the run, CUDA events on the graph's stream */
  uint64_t active[GRE_MAX_RECORDED_SUPERSTEPS];
  /* The plugin's output_statistics (VertexCode.hpp:70), which the engine calls once after the
   * last superstep (Engine.hpp:404), for the gre_vc_* runs: PageRank plugins report the sum of
   * the ranks (Kernels/PageRank.hpp:102-124), ConnectedComponents the number of components
   * (Kernels/CC.hpp:98-120); 0 for the other plugins and the fast paths. */
  double plugin_value;
  uint64_t plugin_count;
} gre_stats;

typedef struct gre_graph_s* gre_graph;

/* ---------------------------------------------------------------------------------------
 * Status and devices
 * ------------------------------------------------------------------------------------- */
/* GRE_Status_Parser::parse (include/Status.hpp:17-30), extended to the added codes. */
const char* gre_status_str(int status);
/* Text of the last error raised on the calling thread ("" if none). */
const char* gre_last_error(void);
/* Number of CUDA devices (0 on a host without GPU). */
int gre_device_count(int* count);
/* Kernels this library has launched so far in the process (its own and the CUB primitives
 * compiled into it).  No reference counterpart: instrumentation for benchmarks. */
uint64_t gre_launch_count(void);

/* ---------------------------------------------------------------------------------------
 * Graph: device CSR (out-arcs) and CSC (in-arcs), uint32 ids, uint64 offsets.
 * Replaces DistributedGraph<GraphInCSR> at one rank (Graph/DistributedGraph.hpp:23-273,
 * Graph/LocalGraph.hpp:23-200).
 * ------------------------------------------------------------------------------------- */
/* DistributedGraph::ingress<dir>(comm, pool, prefix, "ascii", "edgelists")
 * (Graph/DistributedGraph.hpp:153-172; GraphIngress.hpp:76-304,323-328,511-723).
 * `flags` = gre_dir | gre_graph_flags.  Arc order: source-major, file order within a source. */
int gre_graph_load(const char* prefix, uint32_t flags, int device, gre_graph* out);
/* The reference's saved edge partitions (GraphIngress::loadEdgePartitions,
 * GraphIngress.hpp:1024-1071): <prefix>.meta plus <prefix>.part.<nparts>.<r>, r < nparts, each a
 * binary array of (uint64 source, uint64 target) pairs as an np = nparts run wrote them.  All
 * parts are merged into one graph (rank order, file order within a rank); the .outdegree and
 * .scatterMap files are not read (they only serve the exchange between ranks).  Flags as for
 * gre_graph_load. */
int gre_graph_load_parts(const char* prefix, uint32_t nparts, uint32_t flags, int device, gre_graph* out);
/* GraphInCSR::build / rbuild from an edge list in input order (LocalGraph.hpp:66-156). */
int gre_graph_from_edges(uint64_t n, uint64_t m, const uint32_t* src, const uint32_t* dst,
                         uint32_t flags, int device, gre_graph* out);
/* Graph from a CSR (row_off[n+1], col[m]); host or device arrays are copied. */
int gre_graph_from_csr(uint64_t n, uint64_t m, const uint64_t* row_off, const uint32_t* col,
                       uint32_t flags, int device, gre_graph* out);
/* Seeded RMAT graph generated and built on the device (a=.57 b=.19 c=.19), self loops and
 * duplicates removed; symmetric != 0 adds every reverse arc.  Same arcs as gre_rmat_host. */
int gre_graph_rmat(uint32_t scale, uint32_t edgefactor, uint64_t seed, int symmetric, int device,
                   gre_graph* out);
/* Block-diagonal union of k graphs (ids of graph i shifted by vertex_offset[i], written to
 * vertex_offset[0..k], host array).  Runs one launch over many graphs of uneven size. */
int gre_graph_union(const gre_graph* graphs, uint32_t k, int device, gre_graph* out,
                    uint64_t* vertex_offset);
int gre_graph_free(gre_graph g);
/* Relabel the stored graph by decreasing degree (ties by id) so the state of high-degree
 * vertices is packed together and stays cache-resident during random gathers.  Invisible to
 * callers: every entry point keeps taking and returning caller vertex ids, caller vertex order
 * and the arc order of gre_graph_csr.  Plays the role of the reference's local/global id maps
 * (lvid2vid, Graph/DistributedGraph.hpp:57-59).  Graphs built with GRE_GRAPH_REORDER are
 * relabelled on construction.  Arc weights already set are carried along. */
int gre_graph_reorder(gre_graph g);
/* get_num_masters / get_num_edges (DistributedGraph.hpp:93-110). */
int gre_graph_info(gre_graph g, uint64_t* n, uint64_t* m, uint32_t* flags);
/* Threads-per-row schedule of the graph's in-arc (in != 0) or out-arc rows, chosen on first use
 * by the autotuner from the degree distribution (GRE_TUNE=0 in the environment: the default
 * 4 / 4096 / 65536 / 0).  Rows of up to lane_arcs * 2^b arcs get 2^b lanes (b < 5), then a warp
 * up to cta_min arcs, a CTA up to hub_chunk arcs, and chunks of hub_chunk arcs beyond; with
 * seg_window != 0 the rows above cta_min are instead cut at source windows of seg_window
 * vertices and processed window by window.  Replaces the reference's one-thread-per-vertex
 * compute loop (Engine.hpp:592-625), which has no such knob. */
int gre_row_schedule(gre_graph g, int in, uint32_t* lane_arcs, uint64_t* cta_min, uint64_t* hub_chunk,
                     uint64_t* seg_window);
/* getOutdegree for every vertex (DistributedGraph.hpp:178-180). */
int gre_graph_outdegree(gre_graph g, uint32_t* outdeg);
/* Copy the CSR back (row_off[n+1], col[m]) in caller ids; its arc order is the order every
 * per-arc array of this ABI uses (weights, gradients). */
int gre_graph_csr(gre_graph g, uint64_t* row_off, uint32_t* col);
/* DistributedGraph::loadEdgeProperty (DistributedGraph.hpp:195-226): uint32 weight per arc in
 * the arc order of gre_graph_csr. */
int gre_graph_set_weights_u32(gre_graph g, const uint32_t* w);
/* Weight of arc (u,v) = 1 + H(wseed, min(u,v), max(u,v)) % 255 (gre_sssp_weight), computed
 * on the device for every arc. */
int gre_graph_set_weights_hash(gre_graph g, uint64_t wseed);
/* FP64 weight per arc in CSR order (weighted PageRank and its adjoint). */
int gre_graph_set_weights_f64(gre_graph g, const double* w);

/* ---------------------------------------------------------------------------------------
 * Reference-semantics engine: the reference plugins run on a device SynchronousEngine
 * (frontier bitmap + list, combine through atomics, apply on the nextSet bitmap,
 * assert_to_halt).  Per-superstep active counts equal the reference's for deterministic
 * plugins.  `max_supersteps` = configMaxSupersteps (Engine.hpp:148-153; 0 = 1024).
 * ------------------------------------------------------------------------------------- */
/* usr/test_pagerank.cpp: PageRank (variant GRE_PR_REFERENCE) or PageRankIter, run<Out>,
 * srcSet.setALL().  pr: n doubles. */
int gre_vc_pagerank(gre_graph g, int variant, uint32_t max_supersteps, double* pr, gre_stats* st);
/* usr/test_bfs.cpp: BFS plugin (Kernels/BFS.hpp), run<dir> from one source.  pred: n uint64
 * as the plugin leaves it: it forwards pred_scatter = pred (BFS.hpp:66-72), so every reached
 * vertex holds the source's vid and unreached ones UINT64_MAX; level: n int32, the superstep
 * in which apply() reached the vertex (the BFS level; -1 unreached).  Either may be NULL. */
int gre_vc_bfs(gre_graph g, uint32_t src, int dir, uint64_t* pred, int32_t* level, gre_stats* st);
/* usr/test_sssp.cpp: SSSP plugin (Kernels/SSSP.hpp), run<Out>, graph weights required.
 * dist: n uint32 (UINT32_MAX unreached). */
int gre_vc_sssp(gre_graph g, uint32_t src, uint32_t max_supersteps, uint32_t* dist, gre_stats* st);
/* usr/test_cc.cpp: ConnectedComponents (Kernels/CC.hpp), run<InOut>, setALL.  label: n
 * uint32 = minimum vid of the component. */
int gre_vc_cc(gre_graph g, uint32_t* label, gre_stats* st);
/* Kernels/PageRank.hpp:129-197 (PageRank_delta): only rank changes propagate; a vertex stays
 * active while its change exceeds 1e-5.  run<Out> from every vertex; GRE_UNFINISHED when
 * max_supersteps ran out first. */
int gre_vc_pagerank_delta(gre_graph g, uint32_t max_supersteps, double* pr, gre_stats* st);
/* Kernels/SSSP1.hpp:62-95: SSSP with predecessors (pred = the caller id of the vertex whose
 * message set the distance; the source is its own pred, unreached vertices UINT64_MAX with
 * UINT32_MAX distance).  Distances equal the reference's; among predecessors at equal distance
 * the smallest id is kept (the reference keeps whichever message arrived first). */
int gre_vc_sssp1(gre_graph g, uint32_t src, uint32_t max_supersteps, uint32_t* dist, uint64_t* pred,
                 gre_stats* st);
/* Kernels/CountIn.hpp:33-56 with usr/test_cIn.cpp's driver (every vertex active, the reference
 * runs run<In> for one superstep): count[v] = messages v received along `dir`. */
int gre_vc_count_in(gre_graph g, int dir, uint32_t max_supersteps, int32_t* count, gre_stats* st);
/* usr/test_bc.cpp looped over sources: Forward run<Out> + Backward run<In> per level
 * (Kernels/BC.hpp); bc[v] = sum over sources s != v of dep_s(v).  bc: n doubles. */
int gre_vc_bc(gre_graph g, const uint32_t* srcs, uint32_t nsrc, double* bc, gre_stats* st);

/* ---------------------------------------------------------------------------------------
 * B200 fast paths: same results, kernels shaped for the hardware.
 * ------------------------------------------------------------------------------------- */
/* PageRank, pull over in-arcs in FP64, `iters` supersteps, teleport (1-d) (d = 0.85 gives the
 * reference's 0.15).  pr: n doubles. */
int gre_pagerank(gre_graph g, int variant, double d, uint32_t iters, double* pr, gre_stats* st);
/* Direction-optimising BFS, one run per source.  levels: nsrc x n int32 (-1 unreached). */
int gre_bfs(gre_graph g, const uint32_t* srcs, uint32_t nsrc, int32_t* levels, gre_stats* st);
/* No counterpart in the reference.  gre_bfs for callers that cannot let the library allocate
 * device memory (a process whose device memory is reserved and capped by its own pool
 * allocator, or a latency-critical loop that cannot take cudaMalloc's implicit device
 * synchronisation): one source, `level` must be device memory of the graph's device (n int32;
 * anything else: GRE_INVALID_ARG), and all scratch lives in a fixed 32 MiB array inside the
 * library, so graphs are limited to 1,048,576 vertices (larger ones: GRE_INVALID_ARG).  The
 * array is shared by all calls on a device: calls that overlap on the GPU race.  The first call
 * on a device looks up the array's address, and so does the first call after that device's
 * context was replaced (cudaDeviceReset); make those calls before any stream capture. */
int gre_bfs_noalloc(gre_graph g, uint32_t src, int32_t* level, gre_stats* st);
/* Multi-source BFS with 64 sources per uint64 frontier word.  levels: nsrc x n int32. */
int gre_msbfs(gre_graph g, const uint32_t* srcs, uint32_t nsrc, int32_t* levels, gre_stats* st);
/* One BFS whose level-0 frontier holds all `nroots` roots (distance to the nearest root);
 * on a gre_graph_union this is one BFS per member graph in a single launch sequence. */
int gre_bfs_multiroot(gre_graph g, const uint32_t* roots, uint32_t nroots, int32_t* level,
                      gre_stats* st);
/* SSSP with uint32 weights, one run per source.  dist: nsrc x n uint32 (UINT32_MAX
 * unreached).  Graph weights required. */
int gre_sssp(gre_graph g, const uint32_t* srcs, uint32_t nsrc, uint32_t* dist, gre_stats* st);
/* Connected components (symmetric graph): label = minimum vid of the component. */
int gre_cc(gre_graph g, uint32_t* label, gre_stats* st);
/* Brandes betweenness over nsrc sources, bc[v] = sum over s != v of dep_s(v) (FP64).
 * batched = 0: one source at a time; batched = 1: 64 sources per uint64 word.  Both give
 * bit-identical results. */
int gre_bc(gre_graph g, const uint32_t* srcs, uint32_t nsrc, int batched, double* bc, gre_stats* st);
/* Personalised PageRank for k one-hot restart vectors: out[i*n+v], x = (1-d)e_seed + d A^T D^-1 x,
 * `iters` Jacobi steps from x0 = (1-d)e_seed.  batched = 1 runs all k in one pass per step. */
int gre_ppr(gre_graph g, const uint32_t* seeds, uint32_t k, double d, uint32_t iters, int batched,
            double* out, gre_stats* st);
/* Weighted PageRank r = (1-d)pers + d P^T r, P = D_s^-1 W (graph FP64 weights, dangling rows
 * zero), Jacobi steps from r0 = (1-d)pers until max|r_k+1 - r_k| <= tol or max_iters.
 * pers: n doubles (NULL = all ones).  r: n doubles. */
int gre_pagerank_weighted(gre_graph g, double d, const double* pers, double tol, uint32_t max_iters,
                          double* r, gre_stats* st);
/* Adjoint of gre_pagerank_weighted for L = c^T r, given the converged r:
 * lambda = c + d P lambda (same tolerance rule); grad_pers = (1-d) lambda;
 * grad_w[arc u->v] = d r_u / s_u (lambda_v - sum_k P_uk lambda_k) in CSR order.
 * lambda and grad_pers: n doubles (either may be NULL); grad_w: m doubles. */
int gre_pagerank_adjoint(gre_graph g, double d, const double* r, const double* c, double tol,
                         uint32_t max_iters, double* lambda, double* grad_pers, double* grad_w,
                         gre_stats* st);

/* Batches of k graphs of uneven size as one launch sequence: the members' block-diagonal union
 * (gre_graph_union: unrelabelled members, same device) runs the algorithm once, every superstep
 * covering all members; outs[i] receives member i's results (n_i entries, member ids, host or
 * device memory).  Replaces the reference's per-graph driver loop.
 *   GRE_BATCH_BFS       params: uint32_t roots[k] (member ids); outs: int32 levels
 *   GRE_BATCH_CC        params: unused;                        outs: uint32 labels (member ids)
 *   GRE_BATCH_PAGERANK  params: gre_batch_pagerank_params;     outs: double ranks
 * st: the run over the union (its construction is not timed). */
enum gre_batch_algo { GRE_BATCH_BFS = 0, GRE_BATCH_CC = 2, GRE_BATCH_PAGERANK = 3 };
typedef struct {
  int variant; /* gre_pr_variant */
  double d;
  uint32_t iters;
} gre_batch_pagerank_params;
int gre_graph_batch_run(const gre_graph* graphs, uint32_t k, int algo, const void* params,
                        void** outs, gre_stats* st);

/* ---------------------------------------------------------------------------------------
 * 1D-partitioned single-source paths (BFS, PageRank, SSSP, CC): one graph split by vertex over P
 * ranks, one GPU each.
 * Replaces the np > 1 superstep of SynchronousEngine (sync scatters, Engine.hpp:273-315;
 * local compute; sync combiners, Engine.hpp:333-374; apply), with the vertex placement of
 * GraphIngress.hpp:1126-1450 replaced by a fixed one: internal ids dealt to ranks one by one in
 * snake order, L = 64 * ceil(ceil(n / P) / 64) slots per rank.  Each rank keeps the in- and
 * out-arcs of its own vertices.  Results equal the one-GPU calls (levels bit-exact, PageRank
 * with the same per-row association order when the graph's schedule has no source windows).
 * ------------------------------------------------------------------------------------- */
typedef struct gre_part_s* gre_part;

enum gre_exchange_kind {
  GRE_XCHG_ALLGATHER = 0, /* send: `bytes`; recv[q*bytes, (q+1)*bytes) = send of rank q */
  GRE_XCHG_ALLTOALL = 1   /* send: P blocks of `bytes`; recv block q = block `rank` of rank q */
};
/* The collective between the P ranks, supplied by the caller (ncclAllGather / ncclAlltoAll,
 * or torch.distributed).  Every rank calls it the same number of times in the same order.
 * send and recv are device memory of the part's device.  It must run after the work already
 * enqueued on `stream` (the part's cudaStream_t) and complete before work enqueued after it
 * returns: enqueue it on that stream, or synchronise.  Returns 0 on success; anything else
 * ends the call with GRE_FAILURE. */
typedef int (*gre_exchange_fn)(void* ctx, int kind, const void* send, void* recv, uint64_t bytes,
                               void* stream);
/* This rank's part of graph g (on g's device): rows of its slots, columns as exchange indices,
 * row schedule of g.  g may be freed afterwards. */
int gre_part_create(gre_graph g, uint32_t nparts, uint32_t rank, gre_part* out);
int gre_part_free(gre_part p);
/* Slots per rank (L) and arcs of this rank's rows. */
int gre_part_info(gre_part p, uint64_t* slots, uint64_t* arcs_in, uint64_t* arcs_out);
/* Direction-optimising BFS from caller vertex `src`; every rank receives all n levels. */
int gre_part_bfs(gre_part p, uint32_t src, int32_t* level, gre_exchange_fn xchg, void* ctx,
                 gre_stats* st);
/* PageRank as gre_pagerank; every rank receives all n values. */
int gre_part_pagerank(gre_part p, int variant, double d, uint32_t iters, double* pr,
                      gre_exchange_fn xchg, void* ctx, gre_stats* st);

/* SSSP as gre_sssp (uint32 weights the graph had when the part was made); every rank receives
 * all n distances.  Frontier Bellman-Ford supersteps: offers to remote heads go to their owners
 * by one all-to-all per superstep, the owner keeps the smallest. */
int gre_part_sssp(gre_part p, uint32_t src, uint32_t* dist, gre_exchange_fn xchg, void* ctx,
                  gre_stats* st);
/* Connected components as gre_cc (label = smallest caller id of the weak component); every
 * rank receives all n labels.  Label propagation with shortcuts, one all-gather per superstep. */
int gre_part_cc(gre_part p, uint32_t* label, gre_exchange_fn xchg, void* ctx, gre_stats* st);

/* The library's own exchange: NCCL on the part's stream (NCCL is loaded at the first
 * gre_nccl_unique_id / gre_nccl_create: libnccl.so.2 already in the process, else the
 * system's; GRE_NOT_IMPLEMENTED when there is none).  Rank 0 makes the 128-byte id, the host
 * hands it to every rank (any channel), each rank makes its communicator on its device. */
typedef struct gre_nccl_s* gre_nccl;
int gre_nccl_unique_id(uint8_t id[128]);
int gre_nccl_create(const uint8_t id[128], uint32_t nranks, uint32_t rank, int device, gre_nccl* out);
int gre_nccl_free(gre_nccl c);
/* A gre_exchange_fn: pass it with ctx = the gre_nccl of this rank (nranks = the parts). */
int gre_nccl_exchange(void* ctx, int kind, const void* send, void* recv, uint64_t bytes, void* stream);

/* ---------------------------------------------------------------------------------------
 * Host utilities (CPU only, no GPU needed).
 * ------------------------------------------------------------------------------------- */
/* RMAT CSR on the host (same arcs as gre_graph_rmat).  *row_off and *col are malloc'ed;
 * release with gre_host_free. */
int gre_rmat_host(uint32_t scale, uint32_t edgefactor, uint64_t seed, int symmetric, uint64_t* n,
                  uint64_t* m, uint64_t** row_off, uint32_t** col);
void gre_host_free(void* p);
/* Write <prefix>.meta and <prefix>.edges.<i>, i < nfiles, source u in file u % nfiles. */
int gre_write_edgelists(const char* prefix, uint64_t n, uint64_t m, const uint64_t* row_off,
                        const uint32_t* col, uint32_t nfiles);
/* <prefix>.roots: "count\n v1\n v2 ..." (read by Util::loadFromFile, Util/Util.hpp:140-157). */
int gre_write_roots(const char* prefix, const uint32_t* roots, uint32_t count);
int gre_read_roots(const char* prefix, uint32_t* roots, uint32_t capacity, uint32_t* count);
/* Vertex layout of gre_part_create: slots per rank (L) and, when index is not NULL, the
 * exchange index p * L + slot of every internal vertex id v < n (n entries). */
int gre_part_layout(uint64_t n, uint32_t nparts, uint64_t* slots, uint32_t* index);
/* The SSSP weight function of gre_graph_set_weights_hash. */
uint32_t gre_sssp_weight(uint64_t wseed, uint32_t u, uint32_t v);
/* Offline edge partitioner: the reference's single-process EdgePartition::divideEdges
 * (include/Graph/GraphIngress.hpp:1272-1452, usr/debug/test_graphPar.cpp).  Reads <prefix>.meta
 * and the edge lists <prefix>.edges.<i>, places every edge on one of nparts parts by the
 * reference's greedy vertex-cut rule (balance + parts already holding its ends; ties by
 * (u + v) mod ties), and writes <prefix>.part.<nparts>.<r> (the edges as uint64 pairs: what an
 * np = nparts run and gre_graph_load_parts load), <prefix>.outdegree.<nparts>.<p> and
 * <prefix>.scatterMap.<nparts>.<p>.  part_edges (nparts entries, may be NULL) receives the edge
 * count of each part.  nparts in 1..64.  Files are written afresh. */
int gre_partition_edges(const char* prefix, uint32_t nparts, uint64_t* part_edges);

#ifdef __cplusplus
}
#endif
#endif /* GRE_GPU_H */
