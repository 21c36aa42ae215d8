// sssp.cuh -- SSSP app state (internal).
#pragma once
#include "engine.cuh"

namespace mb {

// Default near-far bucket width of a graph: kDeltaWarps warps' worth of
// edges per bucket at the mean degree, times the mean weight.
float sssp_default_delta(const Graph &g);

struct SsspState : FrontierState {
    DevBuf dist, stamp, msg, far[2], farbm, nbm, dprev;
    float default_delta = 0.f;
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
            default_delta = sssp_default_delta(g);
        }
    }
};

// Frontier out-edges from which schedule 0 writes a next-frontier bitmap
// (compacted afterwards) instead of claiming vertices one by one.
// MB_TUNE_SSSP_BM_PUSH_MIN when set, else max(2^20, E/8); 0 turns it off.
uint32_t sssp_bm_push_min(const Context &ctx, const Graph &g);

// One SSSP from `source`; distances are left in st.dist (device).
// phase / force / cont: a run driven one superstep at a time (LoopPhase,
// engine.cuh); the defaults run it whole.
void run_sssp(Context &ctx, Graph &g, SsspState &st, int32_t source, mb_stats *stats, int phase = 0,
             int force = -1, int *cont = nullptr);

}  // namespace mb
