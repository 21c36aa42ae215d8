/*
 * medusa_b200.h -- C ABI of libmedusa_b200.so, the B200 (sm_100a) BSP
 * superstep engine for Medusa's BFS, SSSP and PageRank apps.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes
 * (MB_OK == 0).  Array arguments may be host or device pointers: device
 * pointers are used in place, host pointers are staged through pinned memory.
 * One mb_ctx per host thread; a context owns one CUDA stream and all device
 * scratch; a graph is device-resident until mb_graph_destroy.
 *
 * Sentinels match the reference: BFS unreached level = -1
 * (Algorithm/Message.h:10, Algorithm/main.cu:225-231), SSSP unreached
 * distance = 1e9f (MEDUSA_MAX, SSSP/Configuration.h:6, SSSP/main.cu:324).
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef MEDUSA_B200_H
#define MEDUSA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MB_OK 0
#define MB_ERR_INVALID 1     /* bad argument (null handle, id out of range, ...) */
#define MB_ERR_CUDA 2        /* a CUDA runtime call failed; see mb_last_error */
#define MB_ERR_OOM 3         /* device or pinned allocation failed */
#define MB_ERR_TIMEOUT 4     /* a bounded device-side wait gave up */
#define MB_ERR_UNSUPPORTED 5 /* size or feature outside this build's limits */

/* ---- graph build flags ---------------------------------------------------- */
/* Out-edges of a vertex in input order. */
#define MB_ORDER_INPUT 0u
/* Out-edges of a vertex in reverse input order: the AA order the reference
 * gets from GraphIR::AddEdge prepending (MedusaRT/GraphConverter.cu:191-192)
 * and EdgeArray::buildAA walking each list (SSSP/EdgeDataType.cu:146-157). */
#define MB_ORDER_REFERENCE 1u

/* ---- schedule policies (which kernel runs each superstep) ---------------- */
#define MB_POLICY_FIXED 0       /* the fixed rule: frontier-size thresholds */
#define MB_POLICY_LEARNED 1     /* the trained MLP scheduler, run on the device */
#define MB_POLICY_FORCED 2      /* one schedule id for every superstep */
#define MB_POLICY_ORACLE_BEST 3 /* replay a per-superstep schedule list */

/* Schedule ids.  Every schedule computes identical results; they differ in
 * direction, thread mapping, frontier format and combine fusion only. */
#define MB_SCHED_PUSH_EDGE_QUEUE 0 /* push, edge-balanced (merge-path), queue */
#define MB_SCHED_PUSH_WARP_QUEUE 1 /* push, warp-per-vertex + CTA-per-hub, queue */
#define MB_SCHED_PUSH_EDGE_BITMAP 2 /* push, edge-balanced over a bitmap frontier */
#define MB_SCHED_PUSH_WARP_BITMAP 3 /* push, warp-per-vertex over a bitmap frontier */
#define MB_SCHED_PULL_THREAD 4     /* pull, thread-per-vertex, bitmap frontier */
#define MB_SCHED_PULL_WARP 5       /* pull, warp-per-vertex, bitmap frontier */
#define MB_SCHED_PUSH_UNFUSED 6    /* push into an E-slot message array, then a
                                      separate segmented combine + update (the
                                      reference's send/combine/update split) */
#define MB_SCHED_PULL_UNFUSED 7    /* pull all edges into messages, then combine */
#define MB_NUM_SCHEDULES 8

/* ---- synthetic graph generators ------------------------------------------- */
#define MB_GEN_RMAT 0    /* R-MAT, V = 2^scale, duplicates and self-loops kept */
#define MB_GEN_UNIFORM 1 /* src and dst i.i.d. uniform in [0,V) */
#define MB_GEN_GRID 2    /* rows x cols 4-neighbour grid, bidirectional, with
                            dropped edges and random long-range shortcuts */

typedef struct mb_ctx mb_ctx;
typedef struct mb_graph mb_graph;

typedef struct mb_gen_params {
    int32_t kind;          /* MB_GEN_* */
    int32_t scale;         /* RMAT: V = 2^scale */
    int64_t num_vertices;  /* UNIFORM: V */
    int64_t num_edges;     /* RMAT, UNIFORM: E */
    double a, b, c;        /* RMAT quadrant probabilities (d = 1-a-b-c) */
    int32_t rows, cols;    /* GRID */
    double drop_frac;      /* GRID: fraction of undirected grid edges dropped */
    double shortcut_frac;  /* GRID: shortcut pairs as a fraction of V */
    int32_t wmin, wmax;    /* integer weights in [wmin,wmax] stored as float;
                              wmax == 0: unweighted (all 1) */
    uint64_t seed;
} mb_gen_params;

typedef struct mb_stats {
    int32_t supersteps;        /* BSP supersteps run (for batched runs: max) */
    int32_t status_flags;      /* nonzero: a device-side check tripped */
    int64_t edges_traversed;   /* E_r: sum of out-degrees of reached vertices,
                                  summed over sources (the reference's
                                  traversal count, Algorithm/CPUFunctorHoster.cpp:21) */
    int64_t vertices_reached;  /* summed over sources */
    double device_ms;          /* device time of the superstep loop (CUDA events) */
    int32_t schedule_count[MB_NUM_SCHEDULES]; /* supersteps run per schedule */
    int64_t kernel_launches;   /* kernels this library launched for the call */
    int64_t edges_scanned;     /* edges examined: frontier out-edges of push
                                  supersteps plus E per pull/sweep superstep */
} mb_stats;

/* ---- library / context ---------------------------------------------------- */
const char *mb_version(void);

/* Create a context on CUDA device `device`.
 * Replaces InitConfig + medusaSetDevice + InitCUDA
 * (MultipleGPU/MultiPublicAPI.h:16-39, MultipleGPU/MultiGraphStorage.cu:31-47,
 *  MedusaRT/Utilities.cu:InitCUDA); one GPU only. */
int mb_create(int device, mb_ctx **out);
int mb_destroy(mb_ctx *ctx);
/* Text of the last error on this context (never NULL). */
const char *mb_last_error(const mb_ctx *ctx);
/* Select the per-superstep schedule policy (MB_POLICY_*); `schedule` is the
 * schedule id for MB_POLICY_FORCED and ignored otherwise. */
int mb_set_schedule_policy(mb_ctx *ctx, int policy, int schedule);
/* Replay a per-superstep schedule list (MB_POLICY_ORACLE_BEST): superstep i
 * runs schedules[i]; supersteps past n run schedules[n-1].  n <= 4096.
 * No reference counterpart (the reference has one fixed schedule). */
int mb_set_schedule_replay(mb_ctx *ctx, const int8_t *schedules, int32_t n);
/* SSSP near-far (delta-stepping) bucket width: vertices whose new distance
 * is below the current threshold are expanded next, the rest wait in a far
 * pile until the threshold (raised by delta each time the near frontier runs
 * dry) passes them.  delta > 0: that width; 0 (the default): plain frontier
 * Bellman-Ford; < 0: 32 x mean weight / mean out-degree of the graph.
 * Distances are identical for every delta.  No reference counterpart (the
 * reference relaxes every edge every superstep, SSSP/CPUFunctorHoster.cpp:58-99). */
int mb_set_sssp_delta(mb_ctx *ctx, float delta);
/* 1 (default): supersteps of schedule 0 whose queue frontier is small (at
 * most 2048 vertices and 8192 out-edges, MB_TUNE_TAIL_EDGES) run in one persistent CTA, several
 * supersteps per launch; 0: every superstep is a grid-wide launch.  Results
 * are identical either way. */
int mb_set_persistent_tail(mb_ctx *ctx, int enable);
/* 1: supersteps of schedules 0 and 4 (and near-far splits) run
 * inside one persistent cooperative grid, many supersteps per launch, with
 * grid barriers between them (bounded waits: MB_ERR_TIMEOUT if one gives up);
 * 0 (the default): one launch per superstep.  Identical results either way. */
int mb_set_persistent_grid(mb_ctx *ctx, int enable);
/* 1 (default): BFS (SSSP) with several sources runs them batched, 64 (32)
 * per traversal with per-vertex source masks -- one edge scan serves every
 * source whose frontier holds its tail; 0: one traversal per source.
 * Identical results either way.  No reference counterpart. */
int mb_set_batching(mb_ctx *ctx, int enable);
/* 1: run whole iteration loops as CUDA graphs with device-side convergence
 * (no host round trip per superstep); 0: host-driven loop, one flag read per
 * superstep, as the reference's ResetToExecute/RetriveToExecute loop
 * (MultipleGPU/MultiUtilities.h:48-69). */
int mb_set_graph_capture(mb_ctx *ctx, int enable);

/* ---- graph storage ----------------------------------------------------------- */
/* Build a device-resident graph (CSR + reverse CSR + message slots) from an
 * edge list in insertion order.  w may be NULL (unweighted).
 * Replaces GTGraph::get_parition's single-partition path + GraphIR::AddEdge +
 * InitHostDS + InitDeviceDS (MultipleGPU/PartitionManager.cu:116-534,
 * MedusaRT/GraphConverter.cu:180-196, MultipleGPU/MultiPublicAPI.h:43-96,144-308)
 * and EdgeArray::buildAA / VertexArray::build (SSSP/EdgeDataType.cu:138-186,
 * SSSP/VertexDataType.cu:64-85). */
int mb_graph_from_edges(mb_ctx *ctx, int32_t num_vertices, int64_t num_edges,
                        const int32_t *src, const int32_t *dst, const float *w,
                        uint32_t flags, mb_graph **out);
/* Build a graph from a caller's CSR: row_ptr[V+1] (row_ptr[0] = 0,
 * non-decreasing, row_ptr[V] = E), col[E] and optional weights w[E] (host or
 * device memory); each row keeps the order given, and the reverse CSR and
 * msgDstID are built on the device.  MB_ERR_INVALID for a bad row_ptr or a
 * column id outside [0, V).  Replaces D_EdgeArray::Fill / D_VertexArray::Fill
 * of the reference's CSR arrays (SSSP/EdgeDataType.cu:364-391,
 * SSSP/VertexDataType.cu:88-160) with the reverse layout built by
 * EdgeArray::buildAA (SSSP/EdgeDataType.cu:138-186). */
int mb_graph_upload(mb_ctx *ctx, int32_t num_vertices, int64_t num_edges, const int32_t *row_ptr,
                    const int32_t *col, const float *w, mb_graph **out);
/* Generate a seeded synthetic graph directly in device memory (no reference
 * counterpart: the reference reads GTgraph files). */
int mb_graph_generate(mb_ctx *ctx, const mb_gen_params *params, uint32_t flags,
                      mb_graph **out);
/* The same generator on the host (CPU), for checking: with src == NULL only
 * *num_edges_out is written (grid graphs have a seeded, data-dependent E). */
int mb_generate_edges_host(const mb_gen_params *params, int32_t *src, int32_t *dst,
                           float *w, int64_t *num_edges_out);
int mb_graph_info(const mb_graph *g, int32_t *num_vertices, int64_t *num_edges);
/* Copy the device layout back (any pointer may be NULL):
 * row[V+1], col[E], w[E] (CSR); rrow[V+1], rcol[E] (reverse CSR);
 * mslot[E] (the reference's msgDstID). Replaces D_EdgeArray/D_VertexArray::Dump. */
int mb_graph_export(mb_ctx *ctx, const mb_graph *g, int32_t *row, int32_t *col,
                    float *w, int32_t *rrow, int32_t *rcol, int32_t *mslot);
int mb_graph_destroy(mb_graph *g);

/* ---- apps (one BSP iteration loop each) ---------------------------------------- */
/* BFS levels from each of nsrc sources: levels_out[s*V + v] (-1 unreached).
 * nsrc > 1 runs the sources batched (64-bit per-vertex source masks).
 * Replaces the BFS app's BSP loop + Medusa_Exec + FunctorHolder<EDGE>
 * (Algorithm/main.cu:284-300, Algorithm/UserOperators.h:17-58,
 *  MultipleGPU/MultiAPIHoster.h:653-679) and D_VertexArray::Dump. */
int mb_bfs(mb_ctx *ctx, const mb_graph *g, const int32_t *sources, int32_t nsrc,
           int32_t *levels_out, mb_stats *stats);
/* SSSP distances from each of nsrc sources: dist_out[s*V + v] (1e9 unreached).
 * Replaces SSSP's BSP loop + Medusa_Exec (InitMessageBuffer, ssspEdgeProcAA,
 * Medusa_Combiner::combineAllDevice with CUDPP_MIN, FunctorHolder<VERTEX>)
 * (SSSP/main.cu:369-382, SSSP/UserOperators.h:10-29,151-168,200-264,
 *  MedusaRT/Combiner.cu:82-142). */
int mb_sssp(mb_ctx *ctx, const mb_graph *g, const int32_t *sources, int32_t nsrc,
            float *dist_out, mb_stats *stats);
/* `iters` PageRank supersteps, rank = 0.15 + 0.85 * sum(rank[u]/outdeg[u]),
 * from a uniform initial rank `init`; rank_out[V].
 * Replaces MPG's BSP loop + Medusa_Exec (InitMessageBuffer, SendMsgMEG,
 * combineAllDevice with CUDPP_ADD, FunctorHolder<VERTEX>)
 * (MPG/main.cu:148-169, MPG/UserOperators.h:16-43,119-144,175-270). */
int mb_pagerank(mb_ctx *ctx, const mb_graph *g, int32_t iters, float init,
                float *rank_out, mb_stats *stats);
/* The same from an initial rank per vertex, init_ranks[V] (host or device):
 * the first superstep sends init_ranks[u] / outdeg[u].  This is what one
 * superstep of the reference's PageRank loop does to the rank attribute it
 * holds (MPG/UserOperators.h:16-43, SendMsg + combiner + UpdateVertex), so a
 * loop of single supersteps gives the same bits as one call of many. */
int mb_pagerank_from(mb_ctx *ctx, const mb_graph *g, int32_t iters, const float *init_ranks,
                     float *rank_out, mb_stats *stats);
/* One BSP superstep of a built-in app, for a host that drives the loop
 * itself as the reference's main.cu does (ResetToExecute; Medusa_Exec;
 * exe = RetriveToExecute; super_step++: SSSP/main.cu:369-382,
 * Algorithm/main.cu:284-300, MPG/main.cu:148-169).  app: MB_APP_BFS,
 * MB_APP_SSSP or MB_APP_PAGERANK.  step 0 starts a run (BFS/SSSP from
 * `source`; PageRank from 1/V) and runs its first superstep; each later call
 * runs the next one.  schedule: -1 for the context's policy, else that
 * schedule for this superstep (PageRank: 0 or 6).  *continue_out = 1 while
 * the traversal needs another superstep (PageRank: always 1; the host stops
 * it).  mb_superstep_result then copies the levels (int32), distances or
 * ranks (float) into out[V] (host or device) with the run's statistics and
 * ends the run.  Each call runs exactly one superstep (the persistent
 * tail and grid, which run several per launch, are off in a stepped run).
 * A stepped run holds the graph's state of that app: any
 * whole-run call on the graph (mb_bfs, ...) ends it.  Results are those of
 * the whole-run calls bit for bit, whatever schedules are forced. */
#define MB_APP_BFS 0
#define MB_APP_SSSP 1
#define MB_APP_PAGERANK 2
int mb_superstep(mb_ctx *ctx, const mb_graph *g, int32_t app, int32_t step, int32_t source,
                 int32_t schedule, int32_t *continue_out);
int mb_superstep_result(mb_ctx *ctx, const mb_graph *g, int32_t app, void *out, mb_stats *stats);
/* PageRank summation order.
 * MB_PR_ORDER_REFERENCE (default): the reference's own MEG layout (vertices
 * sorted by out-degree with std::sort, column-major edge slots,
 * MedusaRT/GraphConverter.cu:136-165, MPG/EdgeDataType.cu:45-131), every
 * vertex's messages folded sequentially in float as the reference's combiner
 * does -- the reference's FP32 result bit for bit.  The fused schedule computes
 * those sequential sums in parallel (an exact integer scan within each binade
 * of the running sum, float adds only where the sum changes binade or meets a
 * rounding tie); the message-reading schedule folds each vertex serially.  The
 * ordering is built on first use per graph (a host sort of V out-degrees).
 * MB_PR_ORDER_FIXED: a fixed parallel order, the same for every schedule -- a
 * sequential fold in AA message-slot order up to 64 in-edges, 4096-edge warp
 * blocks above.  Faster on graphs with large hubs; more accurate than the
 * reference's sequential float sums there, and therefore up to ~2e-4 away
 * from the reference's ranks on a vertex with 3.7e5 in-edges (within 1e-5
 * only on graphs without large hubs).  mb_batch_run and mb_pagerank_noalloc
 * use this order. */
#define MB_PR_ORDER_FIXED 0
#define MB_PR_ORDER_REFERENCE 1
int mb_set_pagerank_order(mb_ctx *ctx, int32_t order);

/* Device layout of a graph, for code compiled against the header-only
 * operator API (include/medusa/medusa.h), whose functor kernels read it in
 * place.  Pointers stay valid until mb_graph_destroy.  row/col/esrc/wt: the
 * CSR in the reference's AA edge order (SSSP/EdgeDataType.cu:138-186; esrc is
 * srcVertexID, wt is null for an unweighted graph); rrow/rcol: the reverse
 * CSR, whose position j is message slot j; mslot: msgDstID; outdeg:
 * edge_count (SSSP/VertexDataType.cu:64-85). */
typedef struct mb_graph_view {
    int32_t num_vertices;
    int64_t num_edges;
    const int32_t *row, *col, *esrc, *rrow, *rcol, *mslot, *outdeg;
    const float *wt;
} mb_graph_view;
int mb_graph_device_view(const mb_graph *g, mb_graph_view *view);

/* Graph from GTgraph text (the reference's on-disk format, read by
 * GTGraph::get_parition, MultipleGPU/PartitionManager.cu:153-213): "c"
 * comment lines, one "p <kind> V E" line, "a <src> <dst> <weight>" edge lines
 * with 1-based ids; edges keep file order (AddEdge order).  The text is
 * parsed on the GPU (one thread per line) and the graph built on the device.
 * text: host or device bytes, len bytes long. */
int mb_graph_from_gtgraph(mb_ctx *ctx, const char *text, int64_t len, uint32_t flags,
                          mb_graph **out);

/* ---- visualisation coordinates, headless ---------------------------------- */
/* The reference renders vertices as quads and edges as lines through OpenGL
 * vertex buffers (MedusaRT/GraphRenderingAPI.cu:33-44 DrawNodes, :69-78
 * DrawEdges).  No graphics stack is used here: the same coordinates are
 * written to caller buffers (host or device).
 * mb_vis_node_quads: pos[2V] (x, y per vertex), radius[V] ->
 *   quads[8V] = (x-r, y+r-1), (x+r-1, y+r-1), (x+r-1, y-r), (x-r, y-r).
 * mb_vis_edge_lines: pos[2V] -> lines[4E] = (pos[src], pos[dst]) per edge in
 *   the graph's edge order (the reference's edge array order). */
int mb_vis_node_quads(mb_ctx *ctx, int32_t num_vertices, const float *pos, const int32_t *radius,
                      float *quads_out);
int mb_vis_edge_lines(mb_ctx *ctx, const mb_graph *g, const float *pos, float *lines_out);

/* ---- many graphs in one launch (no reference counterpart) ----------------- */
/* A batch of independent graphs (reference order), e.g. 256 R-MAT graphs of
 * uneven sizes.  mb_batch_run runs, for every graph, `pr_iters` PageRank
 * supersteps from 1/V (as mb_pagerank in MB_PR_ORDER_FIXED, bit for bit) and
 * then one BFS (as mb_bfs) from
 * sources[i] (nullable: vertex 0), all in ONE persistent cooperative launch
 * fed by a device work queue; each graph is worked by a team of CTAs sized
 * by its edge count.  Outputs are concatenated: graph i's ranks and levels
 * at [vbase[i], vbase[i+1]) (mb_batch_vertex_offsets); host or device. */
typedef struct mb_batch mb_batch;
int mb_batch_generate(mb_ctx *ctx, int32_t n, const mb_gen_params *params, mb_batch **out);
/* The same from the caller's graphs: graph i has num_vertices[i] vertices
 * (>= 1) and the num_edges[i] edges that follow graph i-1's in src / dst
 * (host or device memory; ids local to the graph).  num_vertices and
 * num_edges are host arrays of n entries. */
int mb_graph_upload_batch(mb_ctx *ctx, int32_t n, const int32_t *num_vertices,
                          const int64_t *num_edges, const int32_t *src, const int32_t *dst,
                          mb_batch **out);
int mb_batch_info(const mb_batch *b, int32_t *num_graphs, int64_t *total_vertices,
                  int64_t *total_edges);
int mb_batch_vertex_offsets(const mb_batch *b, int64_t *vbase);
int mb_batch_run(mb_ctx *ctx, mb_batch *b, int32_t pr_iters, const int32_t *sources,
                 float *ranks_out, int32_t *levels_out, mb_stats *stats);
int mb_batch_destroy(mb_batch *b);

/* ---- superstep traces (no reference counterpart) ------------------------- */
/* With tracing on, BFS / SSSP / batched-BFS loops run host-driven and every
 * superstep's branch (its kernels, conversion included) is timed alone with
 * CUDA events; mb_get_trace returns the records of the runs since tracing
 * was turned on (oldest first, up to max). */
typedef struct mb_trace_rec {
    int32_t app;      /* 0 BFS, 1 SSSP, 2 batched BFS */
    int32_t step;     /* superstep number */
    int32_t sched;    /* schedule (MB_SCHED_*; 8: near-far split) */
    int32_t branch;   /* loop branch: schedule, +8 with a frontier conversion, 16 split,
                         17 persistent tail, 18 persistent grid, 19 bitmap-output push */
    uint32_t frontier_vertices;
    uint64_t frontier_edges;
    float ms;
} mb_trace_rec;
int mb_set_tracing(mb_ctx *ctx, int enable);
int mb_get_trace(mb_ctx *ctx, mb_trace_rec *out, int32_t max, int32_t *n_out);

/* ---- tunables (no reference counterpart) --------------------------------- */
/* Launch and routing parameters that change speed, never results; set by
 * the autotuner (medusa_b200/autotune.py) or by hand.  value -1 restores
 * the built-in default. */
#define MB_TUNE_SSSP_BM_PUSH_MIN 0 /* SSSP: frontier out-edges from which schedule 0
                                      writes a bitmap compacted afterwards (0: never);
                                      default max(2^20, E/8) */
#define MB_TUNE_PUSH_BLOCKS_PER_SM 1 /* CTAs per SM of the edge-balanced push kernels
                                        (default 8) */
#define MB_TUNE_VERTEX_BLOCKS_PER_SM 2 /* CTAs per SM of the per-vertex / per-word
                                          kernels (default 8) */
#define MB_TUNE_TAIL_EDGES 3 /* frontier out-edges up to which schedule 0 runs in the
                                persistent single-CTA tail (default and maximum 8192) */
#define MB_TUNE_BATCH_THREADS 4 /* threads per CTA of the many-graph kernel (default 256;
                                   a multiple of 32, 64..1024) */
#define MB_TUNE_BATCH_EDGES_PER_CTA 5 /* many-graph kernel: a graph gets one CTA per this
                                         many edges + vertices (default 65536) */
#define MB_TUNE_PR_LIGHT_VPL 6 /* PageRank: light vertices (in-degree <= 64) per lane of
                                  the fused pull, 1, 2 or 4 (default 2, or 1 when that
                                  would give a resident warp fewer than four groups) */
#define MB_TUNE_PR_SHORT_PAIR 7 /* PageRank: heavy-vertex blocks of <= 512 in-edges
                                   folded at once by one warp, 1, 2 or 4 (default 2) */
#define MB_TUNE_BFS_ALPHA 8 /* BFS fixed rule: bottom-up once frontier out-edges x alpha
                               exceed the unvisited out-edges (default 15; 0: never) */
#define MB_TUNE_BFS_BETA 9 /* BFS fixed rule: back to top-down below V / beta frontier
                              vertices (default 20) */
#define MB_TUNE_BULK_STAGE 10 /* SSSP edge-balanced push: 1 stages each tile's queue
                                 entries into shared memory by bulk copies on the
                                 TMA engine, 0 by the threads' loads (default 0) */
#define MB_TUNE_BFS_GAMMA 11 /* BFS fixed rule: bottom-up only while the frontier has
                                at least E / gamma out-edges (default 16; 0: no floor) */
#define MB_TUNE_PR_HUB_MIN 12 /* PageRank in the reference's order: in-degree above
                                which one CTA sums a vertex by the parallel
                                integer scan (default 2048; at least 64) */
#define MB_TUNE_WAIT_POLLS 13 /* polls before a bounded device wait gives up -- the grid
                                barrier of the persistent kernels, the team barrier of the
                                many-graph kernel, the bulk-copy wait of the staged push
                                (defaults 2^22, 2^24, 2^22); the run then fails with
                                MB_ERR_TIMEOUT.  0 gives up at once: a way to drive the
                                error path.  A bulk copy whose wait gave up is still
                                waited for with the full budget before the CTA moves on */
#define MB_TUNE_STEP_CAP 14 /* superstep cap of the BFS / SSSP loops (default V+4 for BFS,
                              4V+16 for SSSP, V+8 batched BFS); past it MB_ERR_TIMEOUT */
#define MB_TUNE_SMALL_PUSH_EDGES 15 /* frontier out-edges up to which schedule 0 (above the
                                      persistent tail's limits) runs on a grid of two CTAs
                                      per SM instead of the full push grid (default
                                      2 x SMs x 512; 0: never) */
#define MB_TUNE_PR_HUB_CTAS 16 /* PageRank in the reference's order: CTAs of the scans of
                                 the hubs above 16384 in-edges, which run beside the other
                                 kernels (default SMs / 4) */
#define MB_TUNE_SSSP_ASYNC 17 /* SSSP: 1 runs the traversal from a queue frontier as one
                                asynchronous cooperative launch (no superstep barriers:
                                warps relax the dirty vertices below a distance threshold
                                that rises by MB_TUNE_ASYNC_DELTA whenever every warp is
                                idle); 0 the BSP supersteps; default 1 (on graphs with
                                hubs only for the tail, MB_TUNE_ASYNC_BELOW), unless the
                                persistent grid is set; never with a near-far width (the
                                far pile is not the kernel's frontier).  Under
                                MB_POLICY_FIXED and MB_POLICY_LEARNED (it is how schedule
                                0 runs the rest of a traversal; the forced and replay
                                policies name every superstep's schedule), and only on
                                graphs without a negative or NaN weight.  Identical
                                distances */
#define MB_TUNE_ASYNC_DELTA 18 /* width by which the asynchronous SSSP's threshold rises
                                 (default: 24 x mean weight / mean out-degree, at least the
                                 mean weight, on graphs without hubs; 0 -- no threshold --
                                 for the tail on graphs with hubs) */
#define MB_TUNE_ASYNC_BLOCKS_PER_SM 19 /* CTAs of 256 threads per SM of the asynchronous
                                         SSSP (default: as many as fit, at most 8) */
#define MB_TUNE_BFS_ASYNC 20 /* BFS: 1 runs a single-source BFS (MB_POLICY_FIXED or
                               MB_POLICY_LEARNED) as
                               the asynchronous kernel with every weight 1 (levels are
                               hop distances; one cooperative launch); 0 the
                               direction-optimising BSP supersteps; default: 1 on graphs
                               without hubs (largest out-degree <= 64) of at most 6
                               edges per vertex.  Identical levels */
#define MB_TUNE_BFS_ASYNC_DELTA 21 /* threshold step of the asynchronous BFS, in hops
                                     (default 8) */
#define MB_TUNE_ASYNC_BELOW 22 /* > 0: the asynchronous SSSP (when on) takes over only
                                 once the frontier, after reaching this many out-edges,
                                 has fewer -- the large supersteps run as BSP pushes and
                                 the long tail of small ones as one asynchronous launch;
                                 0: from the first superstep; default: 0 on graphs
                                 without hubs (largest out-degree <= 64), else
                                 max(2^18, E/16) */
#define MB_TUNE_MSS_DELTA 23 /* batched SSSP (2..32 sources): near-far width -- the
                               frontier holds only the (vertex, source) pairs below a
                               threshold that rises by this much whenever none is
                               left; 0: plain frontier Bellman-Ford; default: 0.3 x
                               the mean weight on graphs whose largest out-degree is
                               above 64 and at most E/1024, else 0 (and 0 when a
                               weight is negative or NaN) */
#define MB_NUM_TUNABLES 24
int mb_set_tunable(mb_ctx *ctx, int32_t which, int64_t value);
int mb_get_tunable(const mb_ctx *ctx, int32_t which, int64_t *value);

/* ---- learned scheduler (no reference counterpart) ------------------------ */
/* One model per loop kind: single-source BFS and SSSP (8 schedules each;
 * the two apps see the same frontier features but rank the schedules
 * differently) and the batched BFS traversal (push 0 vs pull 4).  Under
 * MB_POLICY_LEARNED each loop uses its model; a loop whose model is
 * untrained stays on the fixed rule. */
#define MB_MODEL_BFS 0
#define MB_MODEL_BATCHED 1
#define MB_MODEL_SSSP 2
/* Timing traces for the learned scheduler.  app: 0 BFS, 1 SSSP, 2 batched
 * BFS from `source` and the 63 vertices after it (mod V).  For every
 * superstep of a fixed-rule traversal, the traversal is replayed with each
 * schedule at that superstep (same choices before it; batched: push and
 * pull only) and timed over that superstep and the 3 after it (fixed rule
 * after the choice), since a choice also sets the next frontier's format.  Writes up to max_samples rows of
 * features[6] (the scheduler inputs) and times[8] (ms; -1: not measured) to
 * host arrays, and (nullable) fixed_sched[1] = the schedule the base run
 * chose there; *n_out = rows written.  The base run follows the fixed rule,
 * or the learned policy when that is the context's policy (traces of the
 * states the trained scheduler itself reaches). */
int mb_scheduler_collect(mb_ctx *ctx, const mb_graph *g, int32_t app, int32_t source,
                         float *features, float *times, int32_t *fixed_sched,
                         int32_t max_samples, int32_t *n_out);
/* Train the scheduler MLP (6-32-32-8, FP32) on the GPU: seeded init, `epochs`
 * full-batch Adam steps at learning rate lr, loss = cross-entropy against a
 * softmax of the negated relative times, each sample weighted by its best
 * time.  Arrays may be host or device.
 * *final_loss (nullable) gets the loss after training.  The weights then
 * serve MB_POLICY_LEARNED; the model also records the range of each feature
 * in the training set, and inside a run it overrides the fixed rule only
 * on supersteps whose features lie in that range. */
int mb_scheduler_train(mb_ctx *ctx, int32_t model, const float *features, const float *times,
                       int32_t n, int32_t epochs, float lr, uint64_t seed, float *final_loss);
/* Number of MLP parameters (row-major w1[32][6], b1[32], w2[32][32], b2[32],
 * w3[8][32], b3[8]). */
int32_t mb_scheduler_num_params(void);
int mb_scheduler_get_weights(mb_ctx *ctx, int32_t model, float *weights);
int mb_scheduler_set_weights(mb_ctx *ctx, int32_t model, const float *weights);
/* Loss and its gradient (means over the n samples, each weighted by its
 * best measured time) for given weights,
 * computed by the training kernels (for checking them against an FP64 CPU
 * implementation). */
int mb_scheduler_grad(mb_ctx *ctx, const float *weights, const float *features,
                      const float *times, int32_t n, float *grad_out, float *loss_out);
/* The schedule the model's weights pick for each of n feature rows (host
 * arrays).  fallback (nullable, host): the rule a run applies, keep
 * fallback[i] (the fixed rule's choice) unless the features lie within the
 * training range (+- 1/32) and the network's best output beats that
 * schedule's output by more than 1.0.  Weights set by
 * mb_scheduler_set_weights have an unbounded range. */
int mb_scheduler_pick(mb_ctx *ctx, int32_t model, const float *features,
                      const int32_t *fallback, int32_t n, int32_t *out);

/* PageRank that allocates no memory, for callers that cannot call cudaMalloc
 * (a host application that owns all GPU memory through its own pool, or a
 * latency-bound caller that cannot accept cudaMalloc/cudaFree's device
 * synchronisation).  No counterpart in the reference.
 * Every array is DEVICE memory owned by the caller: row[V+1] out-edge
 * offsets, rrow[V+1] in-edge offsets, rcol[E] in-edge sources grouped by
 * destination (the reverse CSR), rank_out[V].  Same arithmetic and bits as
 * mb_pagerank.  Scratch is one fixed device array in the library (8 MiB per
 * GPU, held until exit), so num_vertices <= 1048576 (larger: MB_ERR_UNSUPPORTED).
 * The arrays must belong to the current device (managed memory is also
 * accepted); another GPU's memory is MB_ERR_INVALID.  The scratch belongs to
 * the context current at the call: every call looks its address up there
 * (no allocation), and the first call in a context also loads the library's
 * device code, so make that first call before any stream capture.  Runs
 * asynchronously on `stream` (a cudaStream_t; NULL = the default stream).
 * All calls on a device share the scratch: calls that overlap on the GPU
 * race.  One warp sums each vertex with more than 64 in-edges, block after
 * block, so a vertex with millions of in-edges makes each superstep as long
 * as that warp's sum (mb_pagerank spreads such a vertex over many warps).
 * A CUDA error left pending by the caller's earlier calls on this thread is
 * cleared on entry; the call reports its own.  Errors: mb_last_error(NULL). */
int mb_pagerank_noalloc(const int32_t *row, const int32_t *rrow, const int32_t *rcol,
                        int32_t num_vertices, int64_t num_edges, int32_t iters, float init,
                        float *rank_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MEDUSA_B200_H */
