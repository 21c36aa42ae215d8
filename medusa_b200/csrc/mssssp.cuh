// mssssp.cuh -- batched SSSP state (internal).
#pragma once
#include "frontier.cuh"

namespace mb {

struct MsSsspState {
    bool built = false;
    int32_t V = 0;
    int64_t E = 0;
    DevBuf dist, front[2], nxt, touched, qv[2], qo[2], tf[2], ctrl, stats, srcs, out;
    ~MsSsspState() { release(); }
    void release() {
        dist.release(); front[0].release(); front[1].release(); nxt.release(); touched.release();
        for (int i = 0; i < 2; i++) { qv[i].release(); qo[i].release(); tf[i].release(); }
        ctrl.release(); stats.release(); srcs.release(); out.release();
        built = false;
    }
    void ensure(const Graph &g);
};

// SSSP from nsrc <= 32 sources at once; dist_dev[s*V + v] (device memory).
void run_mssssp(Context &ctx, Graph &g, MsSsspState &st, const int32_t *sources, int32_t nsrc,
                float *dist_dev, mb_stats *stats);

}  // namespace mb
