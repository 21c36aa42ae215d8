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
    int32_t nlong = 0;  // items longer than kPrShortItem (the head of the list)
    // light vertices (in-degree <= kPrLight) in id order, with their in-edge
    // sources copied out of the reverse CSR: the fused pull streams only
    // these edges (the heavy vertices' edges never enter its windows)
    DevBuf light_v, light_row, light_col;
    int32_t nlight = 0;
    // the reference's MEG order (built on first use): in-edge sources per
    // destination in MEG slot order, and each CSR edge's slot in it
    bool meg_built = false;
    DevBuf meg_src, meg_slot;
    cudaGraphExec_t exec = nullptr;  // captured run (init + iters supersteps)
    int32_t g_iters = -1, g_sched = -1, g_order = -1;
    uint64_t g_tune = ~0ull;  // tunables generation of the captured run
    float g_init = 0.f;
    ~PrState() { release(); }
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        g_iters = -1;
        rank.release(); contrib[0].release(); contrib[1].release(); msg.release();
        items.release(); hub_v.release(); hub_first.release(); blk_sum.release();
        light_v.release(); light_row.release(); light_col.release();
        meg_src.release(); meg_slot.release();
        meg_built = false;
        built = false;
    }
    void ensure(Context &ctx, const Graph &g);
};

// The reference's MEG message order (GraphIR::sortByDegree +
// EdgeArray::buildMEG, MedusaRT/GraphConverter.cu:136-165, MPG/EdgeDataType.cu:45-131).
void build_meg_order(Context &ctx, const Graph &g, PrState &st);

// `iters` supersteps from a uniform initial rank; the ranks are left in
// st.rank (device).  sched: MB_SCHED_PUSH_UNFUSED runs the reference's
// send/combine split, anything else the fused pull; both give identical bits.
// ctx.pr_order MB_PR_ORDER_REFERENCE: every vertex folds its messages
// sequentially in the reference's MEG slot order (slower on hubs).
void run_pagerank(Context &ctx, Graph &g, PrState &st, int32_t iters, float init, int sched,
                  mb_stats *stats);

}  // namespace mb
