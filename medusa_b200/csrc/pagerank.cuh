// pagerank.cuh -- PageRank app state (internal).
#pragma once
#include "mb_internal.cuh"

namespace mb {

struct PrState {
    bool built = false;
    int32_t V = 0;
    int64_t E = 0;
    DevBuf rank, contrib[2], msg, items, hub_v, hub_first, blk_sum;
    int32_t nitems = 0, nhub = 0;
    cudaGraphExec_t exec = nullptr;  // captured run (init + iters supersteps)
    int32_t g_iters = -1, g_sched = -1;
    float g_init = 0.f;
    ~PrState() { release(); }
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        g_iters = -1;
        rank.release(); contrib[0].release(); contrib[1].release(); msg.release();
        items.release(); hub_v.release(); hub_first.release(); blk_sum.release();
        built = false;
    }
    void ensure(Context &ctx, const Graph &g);
};

// `iters` supersteps from a uniform initial rank; the ranks are left in
// st.rank (device).  sched: MB_SCHED_PUSH_UNFUSED runs the reference's
// send/combine split, anything else the fused pull; both give identical bits.
void run_pagerank(Context &ctx, Graph &g, PrState &st, int32_t iters, float init, int sched,
                  mb_stats *stats);

}  // namespace mb
