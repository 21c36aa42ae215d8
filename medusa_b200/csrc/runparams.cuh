// runparams.cuh -- per-run scheduling parameters shared by every BSP loop
// (single-source engine and batched traversals): written by the host into
// the first bytes of a run's device control block before the run.
#pragma once
#include "mb_internal.cuh"

namespace mb {

constexpr int kMaxReplay = 4096;
// BFS fixed rule: bottom-up needs at least E / 16 frontier out-edges.  On
// B200 this leaves C1/C2/C5 (uniform and R-MAT) unchanged and takes the 1448^2
// grid from 1.50 to 1.17 ms (no late bottom-up steps).
constexpr int kBfsGammaDefault = 16;
// Apps of a run (trace records, scheduler features).
constexpr int APP_BFS = 0, APP_SSSP = 1, APP_MSBFS = 2;

struct RunParams {
    int32_t source;
    int32_t policy;
    int32_t forced;
    int32_t nreplay;
    uint32_t launches;          // kernels launched by this run (device-counted)
    float delta;                // SSSP near-far bucket width (0: plain frontier Bellman-Ford)
    int32_t tail;               // 1: small frontiers run in the persistent single-CTA tail
    int32_t persist;            // 1: schedules 0/4 and splits run in the persistent grid
    int32_t replay_then_fixed;  // replay policy: past the list use the fixed rule (else repeat)
    int32_t max_step;           // >= 0: stop after this superstep (trace collection)
    uint32_t tail_edges;        // schedule 0 frontiers up to this many out-edges run in the tail
    uint32_t bm_push_min;       // SSSP: schedule 0 on a queue frontier with at least this many
                                // out-edges writes a bitmap compacted after (0: never)
    int32_t bfs_alpha;          // BFS fixed rule: go bottom-up when frontier out-edges * alpha
                                // exceed the unvisited out-edges (0: never)
    int32_t bfs_beta;           // BFS fixed rule: back to top-down below V / beta frontier vertices
    int32_t bfs_gamma;          // BFS fixed rule: bottom-up only from E / gamma frontier out-edges (0: any)
    int64_t wait_polls;         // polls before a bounded device wait gives up (-1: each wait's default)
    uint32_t small_push_max;    // schedule 0 frontiers up to this many out-edges use the small grid
    int32_t sssp_async;         // SSSP: schedule 0 on a queue frontier runs the asynchronous kernel
    float async_delta;          // its threshold step (0: no threshold)
    uint32_t async_below;       // > 0: ... only once the frontier, after reaching this many
                                // out-edges, has fewer (the big supersteps stay BSP)
    int8_t replay[kMaxReplay];  // MB_POLICY_ORACLE_BEST: schedule per superstep
};

// Write this run's RunParams (policy, forced schedule, replay list, source,
// SSSP bucket width) to a control block whose first member is RunParams.
void upload_params(Context &ctx, void *ctrl_dev, int32_t source, float delta = 0.f,
                   uint32_t bm_push_min = 0, int32_t sssp_async = 0, float async_delta = 0.f,
                   uint32_t async_below = 0);

}  // namespace mb
