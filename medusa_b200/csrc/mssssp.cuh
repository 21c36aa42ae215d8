// mssssp.cuh -- batched SSSP state (internal).
#pragma once
#include "frontier.cuh"

namespace mb {

struct MsSsspState {
    bool built = false;
    int32_t V = 0;
    int64_t E = 0;
    DevBuf dist, front[2], nxt, touched, qv[2], qo[2], tf[2], ctrl, stats, srcs, out;
    DevBuf far, farl[2];  // near-far buckets: waiting pairs per vertex, far lists
    double mean_w = 0.0;     // mean edge weight (the default bucket width)
    bool weights_ok = true;  // no negative or NaN weight (buckets need it)
    ~MsSsspState() { release(); }
    void release() {
        dist.release(); front[0].release(); front[1].release(); nxt.release(); touched.release();
        for (int i = 0; i < 2; i++) { qv[i].release(); qo[i].release(); tf[i].release(); farl[i].release(); }
        ctrl.release(); stats.release(); srcs.release(); out.release(); far.release();
        built = false;
    }
    void ensure(const Graph &g);
};

// Near-far width of the batched SSSP: MB_TUNE_MSS_DELTA when set, else
// mss_default_delta; 0 (plain frontier Bellman-Ford) when a weight is
// negative or NaN.
float mss_default_delta(const Graph &g, double mean_w);
float mss_delta(const Context &ctx, const Graph &g, const MsSsspState &st);

// SSSP from nsrc <= 32 sources at once; dist_dev[s*V + v] (device memory).
void run_mssssp(Context &ctx, Graph &g, MsSsspState &st, const int32_t *sources, int32_t nsrc,
                float *dist_dev, mb_stats *stats);

}  // namespace mb
