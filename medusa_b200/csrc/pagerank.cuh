// pagerank.cuh -- PageRank app state (internal).
#pragma once
#include "mb_internal.cuh"

namespace mb {

struct PrState {
    bool built = false;
    int32_t V = 0;
    int64_t E = 0;
    DevBuf rank, contrib[2], msg, items, hub_v, hub_first, blk_sum;
    DevBuf init_stage;  // host initial ranks of mb_pagerank_from, staged
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
    // the reference's order computed in parallel (built on first use): light
    // lists copied from the MEG order, the mid vertices' sliced ELL, the hubs
    bool exact_built = false;
    int32_t x_hub_min = 0;  // in-degree above which a vertex is a hub
    DevBuf x_light_v, x_light_row, x_light_col;
    int32_t x_nlight = 0;
    DevBuf sell_v, sell_base, sell_rows, sell_src;
    int32_t ngroups = 0;
    DevBuf x_hub_v;
    int32_t x_nhub = 0;
    int32_t x_nbig = 0;  // hubs [0, x_nbig) have more than kHubBig in-edges
    DevBuf x_stage, stage_off, stage_items;  // the hubs' staged contributions
    int32_t nstage_items = 0;
    // the hub kernel runs on a side stream beside the others (fork / join)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // the sliced-ELL kernel on a second side stream beside the others
    cudaStream_t side2 = nullptr;
    cudaEvent_t ev_fork2 = nullptr, ev_join2 = nullptr;
    // the warp-per-hub scans on a third, beside the big hubs' CTAs
    cudaStream_t side3 = nullptr;
    cudaEvent_t ev_join3 = nullptr;
    cudaGraphExec_t exec = nullptr;  // captured run (init + iters supersteps)
    int32_t g_iters = -1, g_sched = -1, g_order = -1;
    uint64_t g_tune = ~0ull;  // tunables generation of the captured run
    float g_init = 0.f;
    const float *g_init_vec = nullptr;  // the initial rank vector the capture reads
    // the side streams and their fork / join events (once)
    void ensure_streams() {
        if (!side) MB_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        if (!ev_fork) MB_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        if (!ev_join) MB_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        if (!side2) MB_CUDA(cudaStreamCreateWithFlags(&side2, cudaStreamNonBlocking));
        if (!ev_fork2) MB_CUDA(cudaEventCreateWithFlags(&ev_fork2, cudaEventDisableTiming));
        if (!ev_join2) MB_CUDA(cudaEventCreateWithFlags(&ev_join2, cudaEventDisableTiming));
        if (!side3) MB_CUDA(cudaStreamCreateWithFlags(&side3, cudaStreamNonBlocking));
        if (!ev_join3) MB_CUDA(cudaEventCreateWithFlags(&ev_join3, cudaEventDisableTiming));
    }
    ~PrState() { release(); }
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        g_iters = -1;
        rank.release(); contrib[0].release(); contrib[1].release(); msg.release();
        init_stage.release();
        items.release(); hub_v.release(); hub_first.release(); blk_sum.release();
        light_v.release(); light_row.release(); light_col.release();
        meg_src.release(); meg_slot.release();
        meg_built = false;
        release_exact();
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        if (ev_fork2) cudaEventDestroy(ev_fork2);
        if (ev_join2) cudaEventDestroy(ev_join2);
        if (side2) cudaStreamDestroy(side2);
        if (ev_join3) cudaEventDestroy(ev_join3);
        if (side3) cudaStreamDestroy(side3);
        ev_fork = ev_join = ev_fork2 = ev_join2 = ev_join3 = nullptr;
        side = side2 = side3 = nullptr;
        built = false;
    }
    void release_exact() {
        x_light_v.release(); x_light_row.release(); x_light_col.release();
        sell_v.release(); sell_base.release(); sell_rows.release(); sell_src.release();
        x_hub_v.release();
        x_stage.release(); stage_off.release(); stage_items.release();
        exact_built = false;
    }
    void ensure(Context &ctx, const Graph &g);
    // the structures of the parallel reference-order sum (meg order included)
    void ensure_exact(Context &ctx, const Graph &g, int32_t hub_min);
};

// The reference's MEG message order (GraphIR::sortByDegree +
// EdgeArray::buildMEG, MedusaRT/GraphConverter.cu:136-165, MPG/EdgeDataType.cu:45-131).
void build_meg_order(Context &ctx, const Graph &g, PrState &st);

// `iters` supersteps from a uniform initial rank; the ranks are left in
// st.rank (device).  sched: MB_SCHED_PUSH_UNFUSED runs the reference's
// send/combine split, anything else the fused pull; both give identical bits.
// ctx.pr_order MB_PR_ORDER_REFERENCE: every vertex's sum is the reference's
// sequential fold over its MEG slots, bit for bit (the fused pull computes
// it in parallel; the message-reading schedule folds each vertex serially).
// init_vec (device, nullable): initial ranks per vertex instead of `init`.
void run_pagerank(Context &ctx, Graph &g, PrState &st, int32_t iters, float init, int sched,
                  mb_stats *stats, const float *init_vec = nullptr);

}  // namespace mb
