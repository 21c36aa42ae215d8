// msbfs.cuh -- batched BFS state (internal).
#pragma once
#include "frontier.cuh"
#include "loopgraph.cuh"
#include "runparams.cuh"

namespace mb {

struct MsBfsState {
    bool built = false;
    int32_t V = 0;
    int64_t E = 0;
    DevBuf seen, front[2], nxt, touched, qv[2], qo[2], tf[2], ctrl, stats, srcs, out;
    // the loop graph and what it was built for (output buffer, batch size, weights)
    LoopGraph lg;
    const void *key_levels = nullptr;
    int32_t key_nsrc = 0;
    const float *key_mlp = nullptr;
    ~MsBfsState() { release(); }
    void release() {
        lg.reset();
        key_levels = nullptr;
        seen.release(); front[0].release(); front[1].release(); nxt.release(); touched.release();
        for (int i = 0; i < 2; i++) { qv[i].release(); qo[i].release(); tf[i].release(); }
        ctrl.release(); stats.release(); srcs.release(); out.release();
        built = false;
    }
    void ensure(const Graph &g);
};

// BFS from nsrc <= 64 sources at once; levels_dev[s*V + v] (device memory).
// Scheduling follows ctx's policy (the batched model under MB_POLICY_LEARNED).
void run_msbfs(Context &ctx, Graph &g, MsBfsState &st, const int32_t *sources, int32_t nsrc,
               int32_t *levels_dev, mb_stats *stats);

}  // namespace mb
