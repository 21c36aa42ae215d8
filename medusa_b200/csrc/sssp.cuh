// sssp.cuh -- SSSP app state (internal).
#pragma once
#include "engine.cuh"

namespace mb {

// Mean edge weight of a graph, and whether any weight is negative or NaN.
void sssp_weight_stats(const Graph &g, double *mean_w, bool *bad);
// Default near-far bucket width of a graph: kDeltaWarps warps' worth of
// edges per bucket at the mean degree, times the mean weight.
float sssp_default_delta(const Graph &g, double mean_w);
// Default threshold step of the asynchronous SSSP: 24 x mean weight / mean
// out-degree, at least the mean weight.
float sssp_async_delta(const Graph &g, double mean_w);

// Shared state of the asynchronous SSSP kernel (sssp.cu), one per run,
// zeroed by the run's init kernel.  Every counter sits on its own 128-byte
// line: the work counters are spread over kAsyncSlots lines so that the
// warps' atomics do not queue on one address.
constexpr int kAsyncSlots = 32;
struct alignas(128) AsyncLine {
    unsigned long long v;
    unsigned long long pad_[15];
};
struct AsyncState {
    AsyncLine p[kAsyncSlots];  // monotone: dirty bits a warp may set, added before it sets any
    AsyncLine d[kAsyncSlots];  // monotone: the part of that it did not set, plus finished claims
    AsyncLine pt;              // (phase << 32) | float bits of the threshold (phase 0: the start's)
    AsyncLine idle[2];         // CTAs whose warps all went idle in the phase of that parity
    AsyncLine mn[2];           // least distance seen above the threshold in that phase (float bits)
    AsyncLine t0;              // least distance of the starting frontier (float bits)
    AsyncLine bar;             // start barrier: CTAs arrived
    AsyncLine abort_;          // nonzero: a wait gave up and every warp leaves
};

struct SsspState : FrontierState {
    DevBuf dist, stamp, msg, far[2], farbm, nbm, dprev, as;
    // hub chunks of the asynchronous kernel, made on its first run on the
    // graph (nchunks < 0: not yet): dirty bitmap over V + 32 * nc32 ids, the
    // first chunk of each hub, each chunk position's hub and first out-edge
    DevBuf adirty, hub_cbase, chunk_src, chunk_rs;
    int64_t nchunks = -1;
    int32_t nc32 = 0;  // chunk c sits at id V + (c % 32) * nc32 + c / 32
    float default_delta = 0.f;
    float async_delta = 0.f;
    bool weights_ok = true;  // no negative or NaN weight (the asynchronous kernel needs it)
    ~SsspState() { release(); }
    void release() {
        release_frontier();
        dist.release();
        stamp.release();
        msg.release();
        far[0].release();
        far[1].release();
        farbm.release();
        nbm.release();
        dprev.release();
        as.release();
        release_chunks();
    }
    void release_chunks() {
        adirty.release();
        hub_cbase.release();
        chunk_src.release();
        chunk_rs.release();
        nchunks = -1;
        nc32 = 0;
    }
    void ensure(const Graph &g) {
        if (ensure_frontier(g)) {
            dist.release();
            stamp.release();
            msg.release();
            dist.reserve(sizeof(float) * (size_t)g.V);
            stamp.reserve(sizeof(int32_t) * (size_t)g.V);
            // E-slot message array of the unfused schedule (the reference's
            // MessageArray, MultipleGPU/MultiPublicAPI.h:178-199)
            msg.reserve(sizeof(float) * (size_t)std::max<int64_t>(g.E, 1));
            far[0].reserve(sizeof(int32_t) * (size_t)g.V);
            far[1].reserve(sizeof(int32_t) * (size_t)g.V);
            farbm.reserve(sizeof(uint32_t) * (size_t)W);
            nbm.reserve(sizeof(uint32_t) * (size_t)W);
            dprev.reserve(sizeof(float) * (size_t)g.V);
            as.reserve(sizeof(AsyncState));
            release_chunks();
            double mean_w = 0.0;
            bool bad = false;
            sssp_weight_stats(g, &mean_w, &bad);
            default_delta = sssp_default_delta(g, mean_w);
            async_delta = sssp_async_delta(g, mean_w);
            weights_ok = !bad;
        }
    }
};

// Graphs without hubs (largest out-degree <= 64): MB_TUNE_SSSP_ASYNC = -1
// runs the whole SSSP in the asynchronous kernel (on other graphs only the
// tail after the frontier's peak, MB_TUNE_ASYNC_BELOW), unless near-far
// buckets or the persistent grid were asked for.  MB_TUNE_BFS_ASYNC = -1:
// the kernel for BFS on hub-free graphs that are also sparse (mean
// out-degree <= 6).  Measured on B200 (ms, BSP -> asynchronous):
// SSSP on the 1448^2 grid 2.5 -> 1.2, uniform 2^20 / 2^24 1.19 -> 0.74,
// uniform 2^18 / 2^22 0.64 -> 0.43; BFS on the grid 1.34 -> 0.72, uniform
// 2^20 with 4 edges per vertex 0.31 -> 0.27, but uniform 2^20 / 2^24 0.21 ->
// 0.29 (the direction-optimising pulls skip most edges).  On R-MAT graphs
// (hubs) the BSP supersteps are as fast or faster for both.
inline bool async_by_default(const Graph &g, bool bfs) {
    if (g.V <= 0 || g.max_outdeg > 64) return false;
    return !bfs || (double)g.E <= 6.0 * (double)g.V;
}

// Frontier out-edges from which schedule 0 writes a next-frontier bitmap
// (compacted afterwards) instead of claiming vertices one by one.
// MB_TUNE_SSSP_BM_PUSH_MIN when set, else max(2^20, E/8); 0 turns it off.
uint32_t sssp_bm_push_min(const Context &ctx, const Graph &g);

// One SSSP from `source`; distances are left in st.dist (device).
// phase / force / cont: a run driven one superstep at a time (LoopPhase,
// engine.cuh); the defaults run it whole.
// bfs_levels (device, V entries): instead a BFS from `source` by the
// asynchronous kernel with every weight 1 (whole runs only; the state should
// then serve BFS runs only, so that its loop graph stays the unit-weight one).
// after: queued behind a whole run, before its host synchronisation.
void run_sssp(Context &ctx, Graph &g, SsspState &st, int32_t source, mb_stats *stats, int phase = 0,
             int force = -1, int *cont = nullptr, int32_t *bfs_levels = nullptr,
             const EmitFn *after = nullptr);

}  // namespace mb
