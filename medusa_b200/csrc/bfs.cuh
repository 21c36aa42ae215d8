// bfs.cuh -- BFS app state (internal).
#pragma once
#include "engine.cuh"

namespace mb {

struct BfsState : FrontierState {
    DevBuf level, vis;
    ~BfsState() { release(); }
    void release() {
        release_frontier();
        level.release();
        vis.release();
    }
    void ensure(const Graph &g) {
        if (ensure_frontier(g)) {
            level.release();
            vis.release();
            level.reserve(sizeof(int32_t) * (size_t)g.V);
            vis.reserve(sizeof(uint32_t) * (size_t)W);
        }
    }
};

// One BFS from `source`; levels are left in st.level (device).
// phase / force / cont: a run driven one superstep at a time (LoopPhase,
// engine.cuh); the defaults run it whole.
// after: queued behind a whole run, before its host synchronisation.
void run_bfs(Context &ctx, Graph &g, BfsState &st, int32_t source, mb_stats *stats, int phase = 0,
             int force = -1, int *cont = nullptr, const EmitFn *after = nullptr);

}  // namespace mb
