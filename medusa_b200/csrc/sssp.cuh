// sssp.cuh -- SSSP app state (internal).
#pragma once
#include "engine.cuh"

namespace mb {

struct SsspState : FrontierState {
    DevBuf dist, stamp, msg;
    ~SsspState() { release(); }
    void release() {
        release_frontier();
        dist.release();
        stamp.release();
        msg.release();
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
        }
    }
};

// One SSSP from `source`; distances are left in st.dist (device).
void run_sssp(Context &ctx, Graph &g, SsspState &st, int32_t source, mb_stats *stats);

}  // namespace mb
