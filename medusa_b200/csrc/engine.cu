// engine.cu -- host side of the superstep engine: run parameters and the
// loop driver (one CUDA-graph launch per run, or the host-driven loop).
#include "engine.cuh"

namespace mb {

void upload_params(Context &ctx, void *ctrl_dev, int32_t source, float delta, uint32_t bm_push_min,
                   int32_t sssp_async, float async_delta, uint32_t async_below) {
    static_assert(sizeof(RunParams) <= Context::kCtrlOff, "params staging too small");
    static_assert(sizeof(Ctrl) <= Context::kSmallBytes - Context::kCtrlOff, "ctrl readback too small");
    RunParams *p = (RunParams *)(ctx.pinned_small + Context::kParamsOff);
    p->source = source;
    p->policy = ctx.schedule_policy;
    p->forced = ctx.fixed_schedule < 0 ? 0 : ctx.fixed_schedule;
    p->nreplay = (int32_t)std::min<size_t>(ctx.replay.size(), kMaxReplay);
    p->launches = 0;
    p->delta = delta;
    p->tail = ctx.tail ? 1 : 0;
    p->persist = ctx.persist ? 1 : 0;
    p->replay_then_fixed = ctx.replay_then_fixed ? 1 : 0;
    p->max_step = ctx.max_step;
    p->bm_push_min = bm_push_min;
    p->sssp_async = sssp_async;
    p->async_delta = async_delta;
    p->async_below = async_below;
    p->bfs_alpha = ctx.tunable[MB_TUNE_BFS_ALPHA] >= 0 ? (int32_t)ctx.tunable[MB_TUNE_BFS_ALPHA] : 15;
    p->bfs_beta = ctx.tunable[MB_TUNE_BFS_BETA] > 0 ? (int32_t)ctx.tunable[MB_TUNE_BFS_BETA] : 20;
    p->bfs_gamma = ctx.tunable[MB_TUNE_BFS_GAMMA] >= 0 ? (int32_t)ctx.tunable[MB_TUNE_BFS_GAMMA] : kBfsGammaDefault;
    p->tail_edges = ctx.tunable[MB_TUNE_TAIL_EDGES] >= 0
                        ? (uint32_t)std::min<int64_t>(ctx.tunable[MB_TUNE_TAIL_EDGES], kTailEdges)
                        : kTailEdges;
    p->wait_polls = ctx.tunable[MB_TUNE_WAIT_POLLS] >= 0 ? ctx.tunable[MB_TUNE_WAIT_POLLS] : -1;
    p->small_push_max = (uint32_t)std::min<int64_t>(
        ctx.tunable[MB_TUNE_SMALL_PUSH_EDGES] >= 0 ? ctx.tunable[MB_TUNE_SMALL_PUSH_EDGES]
                                                   : (int64_t)ctx.num_sms * kSmallPushPerSm * kTile,
        0xffffffffll);
    for (int i = 0; i < p->nreplay; i++) p->replay[i] = ctx.replay[i];
    const size_t bytes = offsetof(RunParams, replay) + (size_t)p->nreplay;
    MB_CUDA(cudaMemcpyAsync(ctrl_dev, p, bytes, cudaMemcpyHostToDevice, ctx.stream));
}

int persistent_grid_size(const Context &ctx, const void *kernel, int threads) {
    int per_sm = 0;
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
    if (per_sm < 1) fail(MB_ERR_UNSUPPORTED, "persistent kernel does not fit on an SM");
    return ctx.num_sms * std::min(per_sm, 4);
}

// One superstep of a stepped run (see LoopPhase); the control block stays
// on the device between calls.
static void run_loop_phase(Context &ctx, LoopSpec &sp, mb_stats *stats, int phase, int force, int *cont) {
    cudaStream_t s = ctx.stream;
    const FrontierArgs &fa = sp.fa;
    Ctrl *hc = (Ctrl *)ctx.ctrl_readback();
    if (phase == LOOP_BEGIN) sp.prologue(s);
    if (phase == LOOP_STEP) {
        if (force >= 0) {
            k_force_sched<<<1, 32, 0, s>>>(fa, force);
            MB_CHECK_LAUNCH();
        }
        MB_CUDA(cudaMemcpyAsync(hc, fa.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        if (hc->done) fail(MB_ERR_INVALID, std::string(sp.name) + ": no superstep left to run");
        sp.branch(hc->branch, s);
    }
    if (phase == LOOP_BEGIN || phase == LOOP_STEP) {
        k_select<<<1, 32, 0, s>>>(fa, sp.app, sp.cap, 0, 0, kNumBranches, 0);
        MB_CHECK_LAUNCH();
    }
    if (phase == LOOP_FINISH && sp.epilogue) sp.epilogue(s);
    MB_CUDA(cudaMemcpyAsync(hc, fa.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    if (cont) *cont = hc->done ? 0 : 1;
    if (hc->err & ERR_STEP_CAP) fail(MB_ERR_TIMEOUT, std::string(sp.name) + ": superstep cap reached");
    if (hc->err & ERR_BULK) fail(MB_ERR_TIMEOUT, std::string(sp.name) + ": a bulk copy timed out");
    if (hc->err & ERR_BARRIER)
        fail(MB_ERR_TIMEOUT, std::string(sp.name) + ": a persistent-grid barrier timed out");
    if (hc->err & ERR_ASYNC)
        fail(MB_ERR_TIMEOUT, std::string(sp.name) + ": a wait of the asynchronous kernel timed out");
    if (phase == LOOP_FINISH && stats) {
        *stats = mb_stats{};
        stats->supersteps = hc->supersteps;
        stats->status_flags = hc->err;
        stats->edges_traversed = (int64_t)hc->edges_reached;
        stats->vertices_reached = (int64_t)hc->reached;
        for (int i = 0; i < MB_NUM_SCHEDULES; i++) stats->schedule_count[i] = hc->sched_count[i];
        stats->kernel_launches = hc->p.launches;
        stats->edges_scanned = (int64_t)hc->work;
    }
}

void run_loop(Context &ctx, LoopSpec &sp, mb_stats *stats, int phase, int force, int *cont) {
    if (phase != LOOP_ALL) {
        run_loop_phase(ctx, sp, stats, phase, force, cont);
        return;
    }
    cudaStream_t s = ctx.stream;
    const int nbranch = kNumBranches;
    FrontierState &st = *sp.st;
    const FrontierArgs &fa = sp.fa;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    try {
        if (ctx.use_graphs && !ctx.tracing) {
            if (!st.lg.exec || st.owner != (const void *)&ctx || st.owner_mlp != (const void *)fa.mlp ||
                st.owner_gen != ctx.tune_gen) {
                const int cap = sp.cap, app = sp.app;
                build_loop_graph(
                    st.lg, s, nbranch, sp.prologue,
                    [&](cudaStream_t cs, cudaGraphConditionalHandle hc,
                        cudaGraphConditionalHandle hb) {
                        k_select<<<1, 32, 0, cs>>>(fa, app, cap, hc, hb, nbranch, 1);
                        MB_CHECK_LAUNCH();
                    },
                    sp.branch, sp.epilogue);
                st.owner = &ctx;
                st.owner_mlp = fa.mlp;
                st.owner_gen = ctx.tune_gen;
            }
            MB_CUDA(cudaEventRecord(e0, s));
            MB_CUDA(cudaGraphLaunch(st.lg.exec, s));
            MB_CUDA(cudaEventRecord(e1, s));
        } else {
            MB_CUDA(cudaEventRecord(e0, s));
            sp.prologue(s);
            Ctrl *hc = (Ctrl *)ctx.ctrl_readback();
            cudaEvent_t t0 = nullptr, t1 = nullptr;
            if (ctx.tracing) {
                MB_CUDA(cudaEventCreate(&t0));
                MB_CUDA(cudaEventCreate(&t1));
            }
            for (;;) {
                k_select<<<1, 32, 0, s>>>(fa, sp.app, sp.cap, 0, 0, nbranch, 0);
                MB_CHECK_LAUNCH();
                MB_CUDA(cudaMemcpyAsync(hc, fa.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
                MB_CUDA(cudaStreamSynchronize(s));
                if (hc->done) break;
                if (ctx.tracing) {
                    // time this superstep alone (its branch, conversion included)
                    Context::TraceRec r;
                    r.app = sp.app;
                    r.step = hc->step;
                    r.sched = hc->sched;
                    r.branch = hc->branch;
                    r.n = hc->front_n;
                    r.m = hc->front_m;
                    for (int i = 0; i < 8; i++) r.feat[i] = hc->feat[i];
                    MB_CUDA(cudaEventRecord(t0, s));
                    sp.branch(hc->branch, s);
                    MB_CUDA(cudaEventRecord(t1, s));
                    MB_CUDA(cudaEventSynchronize(t1));
                    MB_CUDA(cudaEventElapsedTime(&r.ms, t0, t1));
                    ctx.trace.push_back(r);
                } else {
                    sp.branch(hc->branch, s);
                }
            }
            if (t0) cudaEventDestroy(t0);
            if (t1) cudaEventDestroy(t1);
            if (sp.epilogue) sp.epilogue(s);
            MB_CUDA(cudaEventRecord(e1, s));
        }
        // the caller's copies and the control block's readback queued right
        // behind the run: one host synchronisation for all (after e1, so not
        // in the device time)
        if (sp.after) sp.after(s);
        Ctrl *hc = (Ctrl *)ctx.ctrl_readback();
        MB_CUDA(cudaMemcpyAsync(hc, fa.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        float ms = 0;
        MB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (hc->err & ERR_STEP_CAP) fail(MB_ERR_TIMEOUT, std::string(sp.name) + ": superstep cap reached");
        if (hc->err & ERR_BULK) fail(MB_ERR_TIMEOUT, std::string(sp.name) + ": a bulk copy timed out");
        if (hc->err & ERR_BARRIER)
            fail(MB_ERR_TIMEOUT, std::string(sp.name) + ": a persistent-grid barrier timed out");
        if (hc->err & ERR_ASYNC)
            fail(MB_ERR_TIMEOUT, std::string(sp.name) + ": a wait of the asynchronous kernel timed out");
        if (stats) {
            stats->supersteps = hc->supersteps;
            stats->status_flags = hc->err;
            stats->edges_traversed = (int64_t)hc->edges_reached;
            stats->vertices_reached = (int64_t)hc->reached;
            stats->device_ms = ms;
            for (int i = 0; i < MB_NUM_SCHEDULES; i++) stats->schedule_count[i] = hc->sched_count[i];
            stats->kernel_launches = hc->p.launches;
            stats->edges_scanned = (int64_t)hc->work;
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

}  // namespace mb
