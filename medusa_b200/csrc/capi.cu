// capi.cu -- the extern "C" boundary of libmedusa_b200.so (include/medusa_b200.h).
//
// Every entry point catches everything and returns a status code; the text
// of the last error is kept per context (and per thread for calls made
// without a usable context).  Array arguments may be host or device pointers.
#include <cstring>
#include <new>
#include "bfs.cuh"
#include "learn.cuh"
#include "msbfs.cuh"
#include "multigraph.cuh"
#include "mssssp.cuh"
#include "pagerank.cuh"
#include "sched.cuh"
#include "sssp.cuh"

namespace mb {
struct AppStates {
    BfsState bfs;
    SsspState bfs_async;  // the asynchronous BFS's unit-weight runs (MB_TUNE_BFS_ASYNC)
    MsBfsState msbfs;
    SsspState sssp;
    MsSsspState mssssp;
    PrState pr;
    int stepped = -1;  // the app of the stepped run in progress (mb_superstep), or -1
};
int64_t generate_edges_host(const mb_gen_params &p, int32_t *src, int32_t *dst, float *w);
void graph_generate(Context &ctx, Graph &g, const mb_gen_params &p, uint32_t flags);
void vis_node_quads(Context &ctx, int32_t V, const float *pos, const int32_t *radius, float *quads);
void vis_edge_lines(Context &ctx, const Graph &g, const float *pos, float *lines);
}  // namespace mb

struct mb_ctx {
    mb::Context c;
};

struct mb_batch {
    mb::Batch b;
    int device = 0;
};
struct mb_graph {
    mb::Graph g;
};

namespace {

thread_local std::string t_last_error;

int set_error(mb_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->c.last_error = msg;
    t_last_error = msg;
    return code;
}

template <class F>
int guarded(mb_ctx *ctx, F &&f) {
    try {
        f();
        return MB_OK;
    } catch (const mb::ApiError &e) {
        return set_error(ctx, e.code, e.msg);
    } catch (const mb::CudaError &e) {
        std::string m = std::string(cudaGetErrorName(e.err)) + " (" + cudaGetErrorString(e.err) +
                        ") in " + e.what + " at " + e.file + ":" + std::to_string(e.line);
        cudaGetLastError();
        return set_error(ctx, e.err == cudaErrorMemoryAllocation ? MB_ERR_OOM : MB_ERR_CUDA, m);
    } catch (const std::bad_alloc &) {
        return set_error(ctx, MB_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return set_error(ctx, MB_ERR_INVALID, e.what());
    }
}

void use_device(mb_ctx *ctx) { MB_CUDA(cudaSetDevice(ctx->c.device)); }

mb::AppStates &apps(mb_graph *g) {
    if (!g->g.apps) g->g.apps = new mb::AppStates();
    return *g->g.apps;
}

// Copy n int32 from a host or device pointer to host.
std::vector<int32_t> fetch_i32(const int32_t *p, int64_t n) {
    std::vector<int32_t> out((size_t)n);
    if (n > 0) MB_CUDA(cudaMemcpy(out.data(), p, sizeof(int32_t) * (size_t)n, cudaMemcpyDefault));
    return out;
}

void check_graph(mb_ctx *ctx, const mb_graph *g) {
    if (!ctx || !g) mb::fail(MB_ERR_INVALID, "null context or graph");
    if (g->g.device != ctx->c.device) mb::fail(MB_ERR_INVALID, "graph lives on another device");
}

}  // namespace

namespace mb {
// Error text for entry points that have no context (mb_last_error(NULL)).
void record_thread_error(const std::string &msg) { t_last_error = msg; }
}  // namespace mb

extern "C" {

const char *mb_version(void) { return "medusa_b200 0.1 (sm_100a)"; }

int mb_create(int device, mb_ctx **out) {
    if (!out) return set_error(nullptr, MB_ERR_INVALID, "out is null");
    *out = nullptr;
    mb_ctx *ctx = new (std::nothrow) mb_ctx();
    if (!ctx) return set_error(nullptr, MB_ERR_OOM, "host allocation failed");
    int rc = guarded(ctx, [&] {
        int n = 0;
        MB_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) mb::fail(MB_ERR_INVALID, "no such CUDA device");
        MB_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        MB_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10) mb::fail(MB_ERR_UNSUPPORTED, "this build targets sm_100a (B200)");
        ctx->c.device = device;
        ctx->c.num_sms = prop.multiProcessorCount;
        MB_CUDA(cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking));
        MB_CUDA(cudaMallocHost((void **)&ctx->c.pinned_small, mb::Context::kSmallBytes));
        for (mb::DevBuf &b : ctx->c.mlp) {
            b.reserve(sizeof(float) * mb::kModelFloats);
            MB_CUDA(cudaMemsetAsync(b.p, 0, sizeof(float) * mb::kModelFloats, ctx->c.stream));
        }
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
    if (rc != MB_OK) {
        t_last_error = ctx->c.last_error;
        mb_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return MB_OK;
}

int mb_destroy(mb_ctx *ctx) {
    if (!ctx) return MB_OK;
    cudaSetDevice(ctx->c.device);
    if (ctx->c.stream) cudaStreamSynchronize(ctx->c.stream);
    for (auto &b : ctx->c.scratch) b.release();
    for (mb::DevBuf &b : ctx->c.mlp) b.release();
    if (ctx->c.pinned) cudaFreeHost(ctx->c.pinned);
    if (ctx->c.pinned_small) cudaFreeHost(ctx->c.pinned_small);
    if (ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
    delete ctx;
    return MB_OK;
}

const char *mb_last_error(const mb_ctx *ctx) {
    return ctx ? ctx->c.last_error.c_str() : t_last_error.c_str();
}

int mb_set_schedule_policy(mb_ctx *ctx, int policy, int schedule) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    if (policy < MB_POLICY_FIXED || policy > MB_POLICY_ORACLE_BEST)
        return set_error(ctx, MB_ERR_INVALID, "unknown policy");
    if (policy == MB_POLICY_FORCED && (schedule < 0 || schedule >= MB_NUM_SCHEDULES))
        return set_error(ctx, MB_ERR_INVALID, "schedule id out of range");
    if (policy == MB_POLICY_LEARNED && !ctx->c.mlp_ready[MB_MODEL_BFS] &&
        !ctx->c.mlp_ready[MB_MODEL_BATCHED] && !ctx->c.mlp_ready[MB_MODEL_SSSP])
        return set_error(ctx, MB_ERR_INVALID, "the learned scheduler has no weights yet");
    ctx->c.schedule_policy = policy;
    ctx->c.fixed_schedule = schedule;
    return MB_OK;
}

int mb_set_schedule_replay(mb_ctx *ctx, const int8_t *schedules, int32_t n) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    if (n < 1 || n > mb::kMaxReplay || !schedules)
        return set_error(ctx, MB_ERR_INVALID, "replay list must hold 1..4096 schedules");
    for (int32_t i = 0; i < n; i++)
        if (schedules[i] < 0 || schedules[i] >= MB_NUM_SCHEDULES)
            return set_error(ctx, MB_ERR_INVALID, "schedule id out of range");
    ctx->c.replay.assign(schedules, schedules + n);
    ctx->c.schedule_policy = MB_POLICY_ORACLE_BEST;
    ctx->c.fixed_schedule = schedules[n - 1];
    return MB_OK;
}

int mb_set_sssp_delta(mb_ctx *ctx, float delta) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    if (!(delta == delta)) return set_error(ctx, MB_ERR_INVALID, "delta is NaN");
    ctx->c.sssp_delta = delta;
    return MB_OK;
}

int mb_set_persistent_tail(mb_ctx *ctx, int enable) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    ctx->c.tail = enable != 0;
    return MB_OK;
}

int mb_set_persistent_grid(mb_ctx *ctx, int enable) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    ctx->c.persist = enable != 0;
    return MB_OK;
}

namespace {
// n bytes from host or device memory into a device buffer (returns the pointer to use)
const void *stage_in(mb::DevBuf &b, const void *p, size_t n, cudaStream_t s) {
    if (mb::is_device_ptr(p)) return p;
    b.reserve(std::max<size_t>(n, 1));
    mb::copy_sync(s, b.p, p, n);
    return b.p;
}
}  // namespace

int mb_vis_node_quads(mb_ctx *ctx, int32_t V, const float *pos, const int32_t *radius, float *quads) {
    return guarded(ctx, [&] {
        if (!ctx || V < 0 || (V > 0 && (!pos || !radius || !quads))) mb::fail(MB_ERR_INVALID, "bad arguments");
        use_device(ctx);
        mb::DevBuf bp, br, bq;
        const float *dp = (const float *)stage_in(bp, pos, sizeof(float) * 2 * (size_t)V, ctx->c.stream);
        const int32_t *dr = (const int32_t *)stage_in(br, radius, sizeof(int32_t) * (size_t)V, ctx->c.stream);
        float *dq = quads;
        const bool dev_out = mb::is_device_ptr(quads);
        if (!dev_out) dq = (float *)bq.reserve(sizeof(float) * 8 * std::max<size_t>(V, 1));
        mb::vis_node_quads(ctx->c, V, dp, dr, dq);
        if (!dev_out && V)
            MB_CUDA(cudaMemcpyAsync(quads, dq, sizeof(float) * 8 * (size_t)V, cudaMemcpyDeviceToHost, ctx->c.stream));
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

int mb_vis_edge_lines(mb_ctx *ctx, const mb_graph *g, const float *pos, float *lines) {
    return guarded(ctx, [&] {
        check_graph(ctx, g);
        if (!pos || !lines) mb::fail(MB_ERR_INVALID, "bad arguments");
        use_device(ctx);
        mb::DevBuf bp, bl;
        const float *dp = (const float *)stage_in(bp, pos, sizeof(float) * 2 * (size_t)g->g.V, ctx->c.stream);
        float *dl = lines;
        const bool dev_out = mb::is_device_ptr(lines);
        const size_t nb = sizeof(float) * 4 * (size_t)g->g.E;
        if (!dev_out) dl = (float *)bl.reserve(std::max<size_t>(nb, 16));
        mb::vis_edge_lines(ctx->c, g->g, dp, dl);
        if (!dev_out && nb) MB_CUDA(cudaMemcpyAsync(lines, dl, nb, cudaMemcpyDeviceToHost, ctx->c.stream));
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

int mb_set_tracing(mb_ctx *ctx, int enable) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    ctx->c.tracing = enable != 0;
    ctx->c.trace.clear();
    return MB_OK;
}

int mb_get_trace(mb_ctx *ctx, mb_trace_rec *out, int32_t max, int32_t *n_out) {
    if (!ctx || !n_out || max < 0 || (max > 0 && !out)) return set_error(ctx, MB_ERR_INVALID, "bad arguments");
    const int32_t n = (int32_t)std::min<size_t>(ctx->c.trace.size(), (size_t)max);
    for (int32_t i = 0; i < n; i++) {
        const auto &r = ctx->c.trace[i];
        out[i] = mb_trace_rec{r.app, r.step, r.sched, r.branch, r.n, r.m, r.ms};
    }
    *n_out = n;
    return MB_OK;
}

int mb_set_pagerank_order(mb_ctx *ctx, int32_t order) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    if (order != MB_PR_ORDER_FIXED && order != MB_PR_ORDER_REFERENCE)
        return set_error(ctx, MB_ERR_INVALID, "unknown PageRank order");
    ctx->c.pr_order = order;
    return MB_OK;
}

int mb_set_batching(mb_ctx *ctx, int enable) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    ctx->c.batching = enable != 0;
    return MB_OK;
}

int mb_set_graph_capture(mb_ctx *ctx, int enable) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    ctx->c.use_graphs = enable != 0;
    return MB_OK;
}

int mb_set_tunable(mb_ctx *ctx, int32_t which, int64_t value) {
    if (!ctx) return set_error(nullptr, MB_ERR_INVALID, "null context");
    if (which < 0 || which >= MB_NUM_TUNABLES) return set_error(ctx, MB_ERR_INVALID, "unknown tunable");
    if (value < -1) return set_error(ctx, MB_ERR_INVALID, "tunable value must be >= -1");
    if ((which == MB_TUNE_PUSH_BLOCKS_PER_SM || which == MB_TUNE_VERTEX_BLOCKS_PER_SM) &&
        (value == 0 || value > 32))
        return set_error(ctx, MB_ERR_INVALID, "blocks per SM must be 1..32");
    if (which == MB_TUNE_TAIL_EDGES && value > (1 << 24))
        return set_error(ctx, MB_ERR_INVALID, "tail edges must be <= 2^24");
    if (which == MB_TUNE_BATCH_THREADS && value != -1 && (value < 64 || value > 1024 || value % 32))
        return set_error(ctx, MB_ERR_INVALID, "batch threads must be a multiple of 32 in 64..1024");
    if (which == MB_TUNE_BATCH_EDGES_PER_CTA && value == 0)
        return set_error(ctx, MB_ERR_INVALID, "batch edges per CTA must be >= 1");
    if ((which == MB_TUNE_PR_LIGHT_VPL || which == MB_TUNE_PR_SHORT_PAIR) &&
        !(value == -1 || value == 1 || value == 2 || value == 4))
        return set_error(ctx, MB_ERR_INVALID, "PageRank lane/pair counts must be 1, 2 or 4");
    if ((which == MB_TUNE_BFS_ALPHA || which == MB_TUNE_BFS_BETA || which == MB_TUNE_BFS_GAMMA) &&
        value > (1 << 20))
        return set_error(ctx, MB_ERR_INVALID, "BFS alpha / beta must be <= 2^20");
    if (which == MB_TUNE_BFS_BETA && value == 0)
        return set_error(ctx, MB_ERR_INVALID, "BFS beta must be >= 1");
    if (which == MB_TUNE_BULK_STAGE && value > 1)
        return set_error(ctx, MB_ERR_INVALID, "bulk staging is 0 or 1");
    if (which == MB_TUNE_PR_HUB_MIN && value != -1 && (value < 64 || value > 0x7fffffff))
        return set_error(ctx, MB_ERR_INVALID, "PageRank hub threshold must be >= 64");
    if (which == MB_TUNE_SSSP_ASYNC && value > 1)
        return set_error(ctx, MB_ERR_INVALID, "asynchronous SSSP is 0 or 1");
    if (which == MB_TUNE_ASYNC_DELTA && value > (1 << 30))
        return set_error(ctx, MB_ERR_INVALID, "asynchronous SSSP delta must be <= 2^30");
    if (which == MB_TUNE_BFS_ASYNC && value > 1)
        return set_error(ctx, MB_ERR_INVALID, "asynchronous BFS is 0 or 1");
    if (which == MB_TUNE_BFS_ASYNC_DELTA && value > (1 << 30))
        return set_error(ctx, MB_ERR_INVALID, "asynchronous BFS delta must be <= 2^30");
    if (which == MB_TUNE_MSS_DELTA && value > (1 << 30))
        return set_error(ctx, MB_ERR_INVALID, "batched SSSP delta must be <= 2^30");
    if (which == MB_TUNE_ASYNC_BLOCKS_PER_SM && (value == 0 || value > 8))
        return set_error(ctx, MB_ERR_INVALID, "asynchronous SSSP blocks per SM must be 1..8");
    if (ctx->c.tunable[which] == value) return MB_OK;  // nothing to rebuild
    ctx->c.tunable[which] = value;
    ctx->c.tune_gen++;  // captured loop graphs embed launch shapes: rebuild them
    return MB_OK;
}

int mb_get_tunable(const mb_ctx *ctx, int32_t which, int64_t *value) {
    if (!ctx || !value) return set_error(nullptr, MB_ERR_INVALID, "null argument");
    if (which < 0 || which >= MB_NUM_TUNABLES) return MB_ERR_INVALID;
    *value = ctx->c.tunable[which];
    return MB_OK;
}

namespace {
// weights of scheduler model m (MB_MODEL_BFS / MB_MODEL_BATCHED / MB_MODEL_SSSP)
mb::DevBuf &model_weights(mb_ctx *ctx, int32_t m) {
    if (m < 0 || m >= mb::Context::kModels) mb::fail(MB_ERR_INVALID, "unknown scheduler model");
    return ctx->c.mlp[m];
}
bool &model_ready(mb_ctx *ctx, int32_t m) { return ctx->c.mlp_ready[m]; }
// n*k floats from host or device memory into a temporary device buffer
void to_device(mb::DevBuf &b, const float *p, size_t count, cudaStream_t s) {
    b.reserve(sizeof(float) * std::max<size_t>(count, 1));
    mb::copy_sync(s, b.p, p, sizeof(float) * count);
}
}  // namespace

int mb_scheduler_collect(mb_ctx *ctx, const mb_graph *gc, int32_t app, int32_t source,
                         float *features, float *times, int32_t *fixed_sched,
                         int32_t max_samples, int32_t *n_out) {
    return guarded(ctx, [&] {
        check_graph(ctx, gc);
        if (app < 0 || app > 2)
            mb::fail(MB_ERR_INVALID, "app must be 0 (BFS), 1 (SSSP) or 2 (batched BFS)");
        if (!features || !times || !n_out || max_samples < 0) mb::fail(MB_ERR_INVALID, "bad output");
        if (source < 0 || source >= gc->g.V) mb::fail(MB_ERR_INVALID, "source vertex out of range");
        use_device(ctx);
        mb_graph *g = const_cast<mb_graph *>(gc);
        const int a = app == 0 ? mb::APP_BFS : app == 1 ? mb::APP_SSSP : mb::APP_MSBFS;
        *n_out = mb::collect_traces(ctx->c, g->g, apps(g).bfs, apps(g).sssp, apps(g).msbfs, a,
                                    source, features, times, fixed_sched, max_samples);
    });
}

int mb_scheduler_train(mb_ctx *ctx, int32_t model, const float *features, const float *times,
                       int32_t n, int32_t epochs, float lr, uint64_t seed, float *final_loss) {
    return guarded(ctx, [&] {
        if (!ctx) mb::fail(MB_ERR_INVALID, "null context");
        mb::DevBuf &W = model_weights(ctx, model);
        if (n < 1 || !features || !times || epochs < 0 || !(lr > 0.f))
            mb::fail(MB_ERR_INVALID, "bad training arguments");
        use_device(ctx);
        mb::DevBuf X, T;
        to_device(X, features, (size_t)n * mb::kFeat, ctx->c.stream);
        to_device(T, times, (size_t)n * mb::kOut, ctx->c.stream);
        const float loss =
            mb::mlp_train(ctx->c, W.as<float>(), X.as<float>(), T.as<float>(), n, epochs, lr, seed);
        model_ready(ctx, model) = true;
        if (final_loss) *final_loss = loss;
        X.release();
        T.release();
    });
}

int32_t mb_scheduler_num_params(void) { return mb::kMlpParams; }

int mb_scheduler_get_weights(mb_ctx *ctx, int32_t model, float *w) {
    return guarded(ctx, [&] {
        if (!ctx || !w) mb::fail(MB_ERR_INVALID, "null argument");
        use_device(ctx);
        mb::DevBuf &W = model_weights(ctx, model);
        mb::copy_sync(ctx->c.stream, w, W.p, sizeof(float) * mb::kMlpParams);
    });
}

int mb_scheduler_set_weights(mb_ctx *ctx, int32_t model, const float *w) {
    return guarded(ctx, [&] {
        if (!ctx || !w) mb::fail(MB_ERR_INVALID, "null argument");
        use_device(ctx);
        mb::DevBuf &W = model_weights(ctx, model);
        mb::copy_sync(ctx->c.stream, W.p, w, sizeof(float) * mb::kMlpParams);
        mb::mlp_set_open_bounds(ctx->c, W.as<float>());
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
        model_ready(ctx, model) = true;
    });
}

int mb_scheduler_grad(mb_ctx *ctx, const float *weights, const float *features, const float *times,
                      int32_t n, float *grad_out, float *loss_out) {
    return guarded(ctx, [&] {
        if (!ctx || !weights || !features || !times || !grad_out || n < 1)
            mb::fail(MB_ERR_INVALID, "null argument");
        use_device(ctx);
        mb::DevBuf P, X, T, G, L;
        to_device(P, weights, mb::kMlpParams, ctx->c.stream);
        to_device(X, features, (size_t)n * mb::kFeat, ctx->c.stream);
        to_device(T, times, (size_t)n * mb::kOut, ctx->c.stream);
        G.reserve(sizeof(float) * mb::kMlpParams);
        L.reserve(2 * sizeof(float));
        mb::mlp_grad(ctx->c, P.as<float>(), X.as<float>(), T.as<float>(), n, G.as<float>(), L.as<float>());
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
        mb::copy_sync(ctx->c.stream, grad_out, G.p, sizeof(float) * mb::kMlpParams);
        if (loss_out) mb::copy_sync(ctx->c.stream, loss_out, L.p, sizeof(float));
        P.release(); X.release(); T.release(); G.release(); L.release();
    });
}

int mb_scheduler_pick(mb_ctx *ctx, int32_t model, const float *features, const int32_t *fallback,
                      int32_t n, int32_t *out) {
    return guarded(ctx, [&] {
        if (!ctx || !features || !out || n < 0) mb::fail(MB_ERR_INVALID, "null argument");
        use_device(ctx);
        mb::DevBuf &W = model_weights(ctx, model);
        mb::DevBuf X, O, F;
        to_device(X, features, (size_t)n * mb::kFeat, ctx->c.stream);
        O.reserve(sizeof(int32_t) * std::max(n, 1));
        if (fallback) {
            F.reserve(sizeof(int32_t) * std::max(n, 1));
            for (int32_t i = 0; i < n; i++)
                if (fallback[i] < 0 || fallback[i] >= MB_NUM_SCHEDULES)
                    mb::fail(MB_ERR_INVALID, "fallback schedule out of range");
            mb::copy_sync(ctx->c.stream, F.p, fallback, sizeof(int32_t) * n);
        }
        mb::mlp_pick(ctx->c, W.as<float>(), X.as<float>(), fallback ? F.as<int32_t>() : nullptr, n,
                     O.as<int32_t>());
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
        mb::copy_sync(ctx->c.stream, out, O.p, sizeof(int32_t) * n);
        X.release();
        O.release();
        F.release();
    });
}

int mb_graph_from_edges(mb_ctx *ctx, int32_t V, int64_t E, const int32_t *src, const int32_t *dst,
                        const float *w, uint32_t flags, mb_graph **out) {
    if (!ctx || !out) return set_error(ctx, MB_ERR_INVALID, "null context or out");
    *out = nullptr;
    if (V < 1) return set_error(ctx, MB_ERR_INVALID, "num_vertices must be >= 1");
    if (E < 0 || (E > 0 && (!src || !dst))) return set_error(ctx, MB_ERR_INVALID, "bad edge arrays");
    if (E > 0x7FFFFFFFll) return set_error(ctx, MB_ERR_UNSUPPORTED, "num_edges must be < 2^31");
    if (flags & ~MB_ORDER_REFERENCE) return set_error(ctx, MB_ERR_INVALID, "unknown flags");
    mb_graph *g = new (std::nothrow) mb_graph();
    if (!g) return set_error(ctx, MB_ERR_OOM, "host allocation failed");
    int rc = guarded(ctx, [&] {
        use_device(ctx);
        mb::DevBuf bs, bd, bw;
        try {
            const size_t eb = sizeof(uint32_t) * (size_t)std::max<int64_t>(E, 1);
            bs.reserve(eb);
            bd.reserve(eb);
            if (w) bw.reserve(eb);
            if (E > 0) {
                mb::copy_sync(ctx->c.stream, bs.p, src, 4 * (size_t)E);
                mb::copy_sync(ctx->c.stream, bd.p, dst, 4 * (size_t)E);
                if (w) mb::copy_sync(ctx->c.stream, bw.p, w, 4 * (size_t)E);
            }
            mb::graph_build_from_device_edges(ctx->c, g->g, V, E, bs.as<uint32_t>(),
                                              bd.as<uint32_t>(), w ? bw.as<float>() : nullptr, flags);
        } catch (...) {
            bs.release(); bd.release(); bw.release();
            throw;
        }
        bs.release(); bd.release(); bw.release();
    });
    if (rc != MB_OK) {
        mb_graph_destroy(g);
        return rc;
    }
    *out = g;
    return MB_OK;
}

int mb_graph_upload(mb_ctx *ctx, int32_t V, int64_t E, const int32_t *row_ptr, const int32_t *col,
                    const float *w, mb_graph **out) {
    if (!ctx || !out) return set_error(ctx, MB_ERR_INVALID, "null context or out");
    *out = nullptr;
    if (V < 1) return set_error(ctx, MB_ERR_INVALID, "num_vertices must be >= 1");
    if (!row_ptr || E < 0 || (E > 0 && !col)) return set_error(ctx, MB_ERR_INVALID, "bad CSR arrays");
    if (E > 0x7FFFFFFFll) return set_error(ctx, MB_ERR_UNSUPPORTED, "num_edges must be < 2^31");
    mb_graph *g = new (std::nothrow) mb_graph();
    if (!g) return set_error(ctx, MB_ERR_OOM, "host allocation failed");
    int rc = guarded(ctx, [&] {
        use_device(ctx);
        std::vector<int32_t> rp((size_t)V + 1);
        mb::copy_sync(ctx->c.stream, rp.data(), row_ptr, sizeof(int32_t) * rp.size());
        if (rp[0] != 0 || rp[(size_t)V] != E) mb::fail(MB_ERR_INVALID, "row_ptr must run from 0 to num_edges");
        for (int32_t v = 0; v < V; v++)
            if (rp[(size_t)v + 1] < rp[(size_t)v]) mb::fail(MB_ERR_INVALID, "row_ptr must not decrease");
        mb::DevBuf br, bc, bw;
        try {
            const size_t eb = sizeof(uint32_t) * (size_t)std::max<int64_t>(E, 1);
            br.reserve(sizeof(int32_t) * rp.size());
            bc.reserve(eb);
            if (w) bw.reserve(eb);
            mb::copy_sync(ctx->c.stream, br.p, rp.data(), sizeof(int32_t) * rp.size());
            if (E > 0) {
                mb::copy_sync(ctx->c.stream, bc.p, col, 4 * (size_t)E);
                if (w) mb::copy_sync(ctx->c.stream, bw.p, w, 4 * (size_t)E);
            }
            mb::graph_build_from_device_csr(ctx->c, g->g, V, E, br.as<int32_t>(), bc.as<uint32_t>(),
                                            w ? bw.as<float>() : nullptr);
        } catch (...) {
            br.release(); bc.release(); bw.release();
            throw;
        }
        br.release(); bc.release(); bw.release();
    });
    if (rc != MB_OK) {
        mb_graph_destroy(g);
        return rc;
    }
    *out = g;
    return MB_OK;
}

int mb_graph_generate(mb_ctx *ctx, const mb_gen_params *p, uint32_t flags, mb_graph **out) {
    if (!ctx || !out || !p) return set_error(ctx, MB_ERR_INVALID, "null argument");
    *out = nullptr;
    if (flags & ~MB_ORDER_REFERENCE) return set_error(ctx, MB_ERR_INVALID, "unknown flags");
    mb_graph *g = new (std::nothrow) mb_graph();
    if (!g) return set_error(ctx, MB_ERR_OOM, "host allocation failed");
    int rc = guarded(ctx, [&] {
        use_device(ctx);
        if (p->kind != MB_GEN_GRID && p->num_edges > 0x7FFFFFFFll)
            mb::fail(MB_ERR_UNSUPPORTED, "num_edges must be < 2^31");
        mb::graph_generate(ctx->c, g->g, *p, flags);
    });
    if (rc != MB_OK) {
        mb_graph_destroy(g);
        return rc;
    }
    *out = g;
    return MB_OK;
}

int mb_generate_edges_host(const mb_gen_params *p, int32_t *src, int32_t *dst, float *w,
                           int64_t *num_edges_out) {
    if (!p || !num_edges_out) return set_error(nullptr, MB_ERR_INVALID, "null argument");
    return guarded(nullptr, [&] {
        if (src && !dst) mb::fail(MB_ERR_INVALID, "dst is null");
        *num_edges_out = mb::generate_edges_host(*p, src, dst, w);
    });
}

int mb_graph_device_view(const mb_graph *g, mb_graph_view *v) {
    if (!g || !v) return set_error(nullptr, MB_ERR_INVALID, "null argument");
    v->num_vertices = g->g.V;
    v->num_edges = g->g.E;
    v->row = g->g.row.as<int32_t>();
    v->col = g->g.col.as<int32_t>();
    v->esrc = g->g.esrc.as<int32_t>();
    v->rrow = g->g.rrow.as<int32_t>();
    v->rcol = g->g.rcol.as<int32_t>();
    v->mslot = g->g.mslot.as<int32_t>();
    v->outdeg = g->g.outdeg.as<int32_t>();
    v->wt = g->g.weighted ? g->g.wt.as<float>() : nullptr;
    return MB_OK;
}

int mb_graph_from_gtgraph(mb_ctx *ctx, const char *text, int64_t len, uint32_t flags,
                          mb_graph **out) {
    if (!ctx || !out || (!text && len > 0)) return set_error(ctx, MB_ERR_INVALID, "null argument");
    *out = nullptr;
    if (flags & ~MB_ORDER_REFERENCE) return set_error(ctx, MB_ERR_INVALID, "unknown flags");
    mb_graph *g = new (std::nothrow) mb_graph();
    if (!g) return set_error(ctx, MB_ERR_OOM, "host allocation failed");
    int rc = guarded(ctx, [&] {
        use_device(ctx);
        mb::graph_from_gtgraph(ctx->c, g->g, text, len, flags);
        g->g.device = ctx->c.device;
    });
    if (rc != MB_OK) {
        mb_graph_destroy(g);
        return rc;
    }
    *out = g;
    return MB_OK;
}

int mb_graph_info(const mb_graph *g, int32_t *V, int64_t *E) {
    if (!g) return set_error(nullptr, MB_ERR_INVALID, "null graph");
    if (V) *V = g->g.V;
    if (E) *E = g->g.E;
    return MB_OK;
}

int mb_graph_export(mb_ctx *ctx, const mb_graph *g, int32_t *row, int32_t *col, float *w,
                    int32_t *rrow, int32_t *rcol, int32_t *mslot) {
    return guarded(ctx, [&] {
        check_graph(ctx, g);
        use_device(ctx);
        const mb::Graph &G = g->g;
        const size_t vb = sizeof(int32_t) * (size_t)(G.V + 1), eb = sizeof(int32_t) * (size_t)G.E;
        if (row) mb::copy_sync(ctx->c.stream, row, G.row.p, vb);
        if (rrow) mb::copy_sync(ctx->c.stream, rrow, G.rrow.p, vb);
        if (G.E > 0) {
            if (col) mb::copy_sync(ctx->c.stream, col, G.col.p, eb);
            if (w) mb::copy_sync(ctx->c.stream, w, G.wt.p, eb);
            if (rcol) mb::copy_sync(ctx->c.stream, rcol, G.rcol.p, eb);
            if (mslot) mb::copy_sync(ctx->c.stream, mslot, G.mslot.p, eb);
        }
    });
}

int mb_graph_destroy(mb_graph *g) {
    if (!g) return MB_OK;
    cudaSetDevice(g->g.device);
    cudaDeviceSynchronize();
    delete g->g.apps;
    g->g.apps = nullptr;
    g->g.release();
    delete g;
    return MB_OK;
}

int mb_batch_generate(mb_ctx *ctx, int32_t n, const mb_gen_params *params, mb_batch **out) {
    if (!ctx || !out || !params) return set_error(ctx, MB_ERR_INVALID, "null argument");
    *out = nullptr;
    if (n < 1) return set_error(ctx, MB_ERR_INVALID, "a batch holds at least one graph");
    mb_batch *b = new (std::nothrow) mb_batch();
    if (!b) return set_error(ctx, MB_ERR_OOM, "host allocation failed");
    int rc = guarded(ctx, [&] {
        use_device(ctx);
        b->device = ctx->c.device;
        for (int32_t i = 0; i < n; i++)
            if (params[i].kind != MB_GEN_GRID && params[i].num_edges > 0x7FFFFFFFll)
                mb::fail(MB_ERR_UNSUPPORTED, "num_edges must be < 2^31");
        mb::batch_generate(ctx->c, b->b, params, n);
    });
    if (rc != MB_OK) {
        mb_batch_destroy(b);
        return rc;
    }
    *out = b;
    return MB_OK;
}

int mb_graph_upload_batch(mb_ctx *ctx, int32_t n, const int32_t *nv, const int64_t *ne,
                          const int32_t *src, const int32_t *dst, mb_batch **out) {
    if (!ctx || !out || !nv || !ne) return set_error(ctx, MB_ERR_INVALID, "null argument");
    *out = nullptr;
    if (n < 1) return set_error(ctx, MB_ERR_INVALID, "a batch holds at least one graph");
    int64_t total = 0;
    for (int32_t i = 0; i < n; i++) {
        if (nv[i] < 1) return set_error(ctx, MB_ERR_INVALID, "num_vertices must be >= 1");
        if (ne[i] < 0) return set_error(ctx, MB_ERR_INVALID, "num_edges must be >= 0");
        if (ne[i] > 0x7FFFFFFFll) return set_error(ctx, MB_ERR_UNSUPPORTED, "num_edges must be < 2^31");
        total += ne[i];
    }
    if (total > 0 && (!src || !dst)) return set_error(ctx, MB_ERR_INVALID, "bad edge arrays");
    mb_batch *b = new (std::nothrow) mb_batch();
    if (!b) return set_error(ctx, MB_ERR_OOM, "host allocation failed");
    int rc = guarded(ctx, [&] {
        use_device(ctx);
        b->device = ctx->c.device;
        mb::batch_from_edges(ctx->c, b->b, n, nv, ne, src, dst);
    });
    if (rc != MB_OK) {
        mb_batch_destroy(b);
        return rc;
    }
    *out = b;
    return MB_OK;
}

int mb_batch_info(const mb_batch *b, int32_t *num_graphs, int64_t *total_vertices,
                  int64_t *total_edges) {
    if (!b) return set_error(nullptr, MB_ERR_INVALID, "null batch");
    if (num_graphs) *num_graphs = (int32_t)b->b.graphs.size();
    if (total_vertices) *total_vertices = b->b.total_V;
    if (total_edges) *total_edges = b->b.total_E;
    return MB_OK;
}

int mb_batch_vertex_offsets(const mb_batch *b, int64_t *vbase) {
    if (!b || !vbase) return set_error(nullptr, MB_ERR_INVALID, "null argument");
    std::memcpy(vbase, b->b.vbase.data(), sizeof(int64_t) * b->b.vbase.size());
    return MB_OK;
}

int mb_batch_run(mb_ctx *ctx, mb_batch *b, int32_t pr_iters, const int32_t *sources,
                 float *ranks_out, int32_t *levels_out, mb_stats *stats) {
    return guarded(ctx, [&] {
        if (!ctx || !b || !ranks_out || !levels_out) mb::fail(MB_ERR_INVALID, "null argument");
        if (b->device != ctx->c.device) mb::fail(MB_ERR_INVALID, "batch lives on another device");
        if (pr_iters < 0) mb::fail(MB_ERR_INVALID, "pr_iters must be >= 0");
        use_device(ctx);
        const int32_t n = (int32_t)b->b.graphs.size();
        std::vector<int32_t> src;
        if (sources) src = fetch_i32(sources, n);
        const size_t nv = (size_t)b->b.total_V;
        const bool dev_r = mb::is_device_ptr(ranks_out), dev_l = mb::is_device_ptr(levels_out);
        float *r = ranks_out;
        int32_t *l = levels_out;
        if (!dev_r) r = (float *)b->b.rank.reserve(sizeof(float) * std::max<size_t>(nv, 1));
        if (!dev_l) l = (int32_t *)b->b.level.reserve(sizeof(int32_t) * std::max<size_t>(nv, 1));
        mb::batch_run(ctx->c, b->b, pr_iters, sources ? src.data() : nullptr, r, l, stats);
        if (!dev_r) MB_CUDA(cudaMemcpyAsync(ranks_out, r, sizeof(float) * nv, cudaMemcpyDeviceToHost, ctx->c.stream));
        if (!dev_l) MB_CUDA(cudaMemcpyAsync(levels_out, l, sizeof(int32_t) * nv, cudaMemcpyDeviceToHost, ctx->c.stream));
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

int mb_batch_destroy(mb_batch *b) {
    if (!b) return MB_OK;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    b->b.release();
    delete b;
    return MB_OK;
}

int mb_bfs(mb_ctx *ctx, const mb_graph *gc, const int32_t *sources, int32_t nsrc,
           int32_t *levels_out, mb_stats *stats) {
    return guarded(ctx, [&] {
        check_graph(ctx, gc);
        if (nsrc < 1 || !sources || !levels_out) mb::fail(MB_ERR_INVALID, "bad sources/output");
        use_device(ctx);
        mb_graph *g = const_cast<mb_graph *>(gc);
        apps(g).stepped = -1;  // a whole run ends any stepped one
        const int32_t V = g->g.V;
        std::vector<int32_t> src = fetch_i32(sources, nsrc);
        for (int32_t s : src)
            if (s < 0 || s >= V) mb::fail(MB_ERR_INVALID, "source vertex out of range");
        mb_stats total{};
        if (nsrc > 1 && ctx->c.batching) {
            // batches of up to 64 sources, one masked traversal each
            mb::MsBfsState &ms = apps(g).msbfs;
            ms.ensure(g->g);  // before reserving ms.out (a rebuild releases it)
            const bool dev_out = mb::is_device_ptr(levels_out);
            for (int32_t b0 = 0; b0 < nsrc; b0 += 64) {
                const int32_t nb = std::min<int32_t>(64, nsrc - b0);
                int32_t *dst = levels_out + (size_t)b0 * V;
                int32_t *dev = dst;
                if (!dev_out) dev = (int32_t *)ms.out.reserve(sizeof(int32_t) * (size_t)nb * V);
                mb_stats st{};
                mb::run_msbfs(ctx->c, g->g, ms, src.data() + b0, nb, dev, &st);
                if (!dev_out)
                    MB_CUDA(cudaMemcpyAsync(dst, dev, sizeof(int32_t) * (size_t)nb * V,
                                            cudaMemcpyDeviceToHost, ctx->c.stream));
                total.supersteps = std::max(total.supersteps, st.supersteps);
                total.edges_traversed += st.edges_traversed;
                total.vertices_reached += st.vertices_reached;
                total.device_ms += st.device_ms;
                total.kernel_launches += st.kernel_launches;
                for (int k = 0; k < MB_NUM_SCHEDULES; k++) total.schedule_count[k] += st.schedule_count[k];
            }
            MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
            if (stats) *stats = total;
            return;
        }
        const int64_t t_async = ctx->c.tunable[MB_TUNE_BFS_ASYNC];
        const bool bfs_async = (t_async > 0 || (t_async < 0 && mb::async_by_default(g->g, true))) &&
                               (ctx->c.schedule_policy == MB_POLICY_FIXED ||
                                ctx->c.schedule_policy == MB_POLICY_LEARNED) &&
                               !ctx->c.persist;
        if (bfs_async) apps(g).bfs.ensure(g->g);
        for (int32_t i = 0; i < nsrc; i++) {
            mb_stats st{};
            // the levels' copy out rides on the run's own synchronisation
            const mb::EmitFn copy_out = [&](cudaStream_t s) {
                MB_CUDA(cudaMemcpyAsync(levels_out + (size_t)i * V, apps(g).bfs.level.p,
                                        sizeof(int32_t) * (size_t)V, cudaMemcpyDefault, s));
            };
            if (bfs_async)
                mb::run_sssp(ctx->c, g->g, apps(g).bfs_async, src[i], &st, mb::LOOP_ALL, -1, nullptr,
                             apps(g).bfs.level.as<int32_t>(), &copy_out);
            else
                mb::run_bfs(ctx->c, g->g, apps(g).bfs, src[i], &st, mb::LOOP_ALL, -1, nullptr, &copy_out);
            total.supersteps = std::max(total.supersteps, st.supersteps);
            total.status_flags |= st.status_flags;
            total.edges_traversed += st.edges_traversed;
            total.vertices_reached += st.vertices_reached;
            total.device_ms += st.device_ms;
            for (int k = 0; k < MB_NUM_SCHEDULES; k++) total.schedule_count[k] += st.schedule_count[k];
            total.kernel_launches += st.kernel_launches;
            total.edges_scanned += st.edges_scanned;
        }
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
        if (stats) *stats = total;
    });
}

int mb_sssp(mb_ctx *ctx, const mb_graph *gc, const int32_t *sources, int32_t nsrc, float *dist_out,
            mb_stats *stats) {
    return guarded(ctx, [&] {
        check_graph(ctx, gc);
        if (nsrc < 1 || !sources || !dist_out) mb::fail(MB_ERR_INVALID, "bad sources/output");
        use_device(ctx);
        mb_graph *g = const_cast<mb_graph *>(gc);
        apps(g).stepped = -1;  // a whole run ends any stepped one
        const int32_t V = g->g.V;
        std::vector<int32_t> src = fetch_i32(sources, nsrc);
        for (int32_t s : src)
            if (s < 0 || s >= V) mb::fail(MB_ERR_INVALID, "source vertex out of range");
        mb_stats total{};
        if (nsrc > 1 && ctx->c.batching) {
            // batches of up to 32 sources, one masked traversal each
            mb::MsSsspState &ms = apps(g).mssssp;
            ms.ensure(g->g);  // before reserving ms.out (a rebuild releases it)
            const bool dev_out = mb::is_device_ptr(dist_out);
            for (int32_t b0 = 0; b0 < nsrc; b0 += 32) {
                const int32_t nb = std::min<int32_t>(32, nsrc - b0);
                float *dst = dist_out + (size_t)b0 * V;
                float *dev = dst;
                if (!dev_out) dev = (float *)ms.out.reserve(sizeof(float) * (size_t)nb * V);
                mb_stats st{};
                mb::run_mssssp(ctx->c, g->g, ms, src.data() + b0, nb, dev, &st);
                if (!dev_out)
                    MB_CUDA(cudaMemcpyAsync(dst, dev, sizeof(float) * (size_t)nb * V,
                                            cudaMemcpyDeviceToHost, ctx->c.stream));
                total.supersteps = std::max(total.supersteps, st.supersteps);
                total.edges_traversed += st.edges_traversed;
                total.vertices_reached += st.vertices_reached;
                total.device_ms += st.device_ms;
                total.kernel_launches += st.kernel_launches;
                total.edges_scanned += st.edges_scanned;
                for (int k = 0; k < MB_NUM_SCHEDULES; k++) total.schedule_count[k] += st.schedule_count[k];
            }
            MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
            if (stats) *stats = total;
            return;
        }
        for (int32_t i = 0; i < nsrc; i++) {
            mb_stats st{};
            // the distances' copy out rides on the run's own synchronisation
            const mb::EmitFn copy_out = [&](cudaStream_t s) {
                MB_CUDA(cudaMemcpyAsync(dist_out + (size_t)i * V, apps(g).sssp.dist.p,
                                        sizeof(float) * (size_t)V, cudaMemcpyDefault, s));
            };
            mb::run_sssp(ctx->c, g->g, apps(g).sssp, src[i], &st, mb::LOOP_ALL, -1, nullptr, nullptr, &copy_out);
            total.supersteps = std::max(total.supersteps, st.supersteps);
            total.status_flags |= st.status_flags;
            total.edges_traversed += st.edges_traversed;
            total.vertices_reached += st.vertices_reached;
            total.device_ms += st.device_ms;
            for (int k = 0; k < MB_NUM_SCHEDULES; k++) total.schedule_count[k] += st.schedule_count[k];
            total.kernel_launches += st.kernel_launches;
            total.edges_scanned += st.edges_scanned;
        }
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
        if (stats) *stats = total;
    });
}

int mb_pagerank(mb_ctx *ctx, const mb_graph *gc, int32_t iters, float init, float *rank_out,
                mb_stats *stats) {
    return guarded(ctx, [&] {
        check_graph(ctx, gc);
        if (iters < 0 || !rank_out) mb::fail(MB_ERR_INVALID, "bad iters/output");
        use_device(ctx);
        mb_graph *g = const_cast<mb_graph *>(gc);
        apps(g).stepped = -1;  // a whole run ends any stepped one
        const int sched = ctx->c.schedule_policy == MB_POLICY_FORCED ? ctx->c.fixed_schedule
                                                                      : MB_SCHED_PUSH_EDGE_QUEUE;
        mb::run_pagerank(ctx->c, g->g, apps(g).pr, iters, init, sched, stats);
        MB_CUDA(cudaMemcpyAsync(rank_out, apps(g).pr.rank.p, sizeof(float) * (size_t)g->g.V,
                                cudaMemcpyDefault, ctx->c.stream));
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

int mb_superstep(mb_ctx *ctx, const mb_graph *gc, int32_t app, int32_t step, int32_t source,
                 int32_t schedule, int32_t *continue_out) {
    return guarded(ctx, [&] {
        check_graph(ctx, gc);
        if (!continue_out || step < 0) mb::fail(MB_ERR_INVALID, "bad step/output");
        if (schedule < -1 || schedule >= MB_NUM_SCHEDULES) mb::fail(MB_ERR_INVALID, "bad schedule");
        use_device(ctx);
        mb_graph *g = const_cast<mb_graph *>(gc);
        mb::AppStates &as = apps(g);
        int cont = 0;
        if (app == MB_APP_BFS || app == MB_APP_SSSP) {
            if (step == 0 && (source < 0 || source >= g->g.V)) mb::fail(MB_ERR_INVALID, "source vertex out of range");
            if (step > 0 && as.stepped != app) mb::fail(MB_ERR_INVALID, "no stepped run of this app in progress");
            // step 0 starts the run and picks its first superstep, then runs it
            if (step == 0) {
                if (app == MB_APP_BFS) mb::run_bfs(ctx->c, g->g, as.bfs, source, nullptr, mb::LOOP_BEGIN, -1, &cont);
                else mb::run_sssp(ctx->c, g->g, as.sssp, source, nullptr, mb::LOOP_BEGIN, -1, &cont);
                as.stepped = app;
            }
            if (step == 0 && !cont) {
                *continue_out = 0;
                return;
            }
            if (app == MB_APP_BFS) mb::run_bfs(ctx->c, g->g, as.bfs, 0, nullptr, mb::LOOP_STEP, schedule, &cont);
            else mb::run_sssp(ctx->c, g->g, as.sssp, 0, nullptr, mb::LOOP_STEP, schedule, &cont);
        } else if (app == MB_APP_PAGERANK) {
            if (schedule != -1 && schedule != MB_SCHED_PUSH_EDGE_QUEUE && schedule != MB_SCHED_PUSH_UNFUSED)
                mb::fail(MB_ERR_INVALID, "PageRank schedules are 0 and 6");
            if (step > 0 && as.stepped != app) mb::fail(MB_ERR_INVALID, "no stepped run of this app in progress");
            const int sched = schedule == MB_SCHED_PUSH_UNFUSED ? MB_SCHED_PUSH_UNFUSED : MB_SCHED_PUSH_EDGE_QUEUE;
            mb::PrState &pr = as.pr;
            if (step == 0) mb::run_pagerank(ctx->c, g->g, pr, 1, 1.0f / (float)g->g.V, sched, nullptr);
            else mb::run_pagerank(ctx->c, g->g, pr, 1, 0.f, sched, nullptr, pr.rank.as<float>());
            as.stepped = app;
            cont = 1;  // the host decides how many supersteps PageRank runs
        } else {
            mb::fail(MB_ERR_INVALID, "unknown app");
        }
        *continue_out = cont;
    });
}

int mb_superstep_result(mb_ctx *ctx, const mb_graph *gc, int32_t app, void *out, mb_stats *stats) {
    return guarded(ctx, [&] {
        check_graph(ctx, gc);
        if (!out) mb::fail(MB_ERR_INVALID, "null output");
        use_device(ctx);
        mb_graph *g = const_cast<mb_graph *>(gc);
        mb::AppStates &as = apps(g);
        if (as.stepped != app) mb::fail(MB_ERR_INVALID, "no stepped run of this app");
        const size_t bytes = 4 * (size_t)g->g.V;
        const void *src = nullptr;
        if (app == MB_APP_BFS) {
            mb::run_bfs(ctx->c, g->g, as.bfs, 0, stats, mb::LOOP_FINISH);
            src = as.bfs.level.p;
        } else if (app == MB_APP_SSSP) {
            mb::run_sssp(ctx->c, g->g, as.sssp, 0, stats, mb::LOOP_FINISH);
            src = as.sssp.dist.p;
        } else {
            src = as.pr.rank.p;
            if (stats) *stats = mb_stats{};
        }
        MB_CUDA(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDefault, ctx->c.stream));
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
        as.stepped = -1;
    });
}

int mb_pagerank_from(mb_ctx *ctx, const mb_graph *gc, int32_t iters, const float *init_ranks,
                     float *rank_out, mb_stats *stats) {
    return guarded(ctx, [&] {
        check_graph(ctx, gc);
        if (iters < 0 || !rank_out || !init_ranks) mb::fail(MB_ERR_INVALID, "bad iters/input/output");
        use_device(ctx);
        mb_graph *g = const_cast<mb_graph *>(gc);
        apps(g).stepped = -1;  // a whole run ends any stepped one
        const int sched = ctx->c.schedule_policy == MB_POLICY_FORCED ? ctx->c.fixed_schedule
                                                                      : MB_SCHED_PUSH_EDGE_QUEUE;
        // host ranks are staged into the PageRank state's own buffer, so a
        // captured run keeps reading the same address
        mb::PrState &pr = apps(g).pr;
        const size_t bytes = sizeof(float) * (size_t)g->g.V;
        const float *init_dev = init_ranks;
        if (!mb::is_device_ptr(init_ranks)) {
            pr.init_stage.reserve(std::max<size_t>(bytes, 1));
            mb::copy_sync(ctx->c.stream, pr.init_stage.p, init_ranks, bytes);
            init_dev = pr.init_stage.as<float>();
        }
        mb::run_pagerank(ctx->c, g->g, pr, iters, 0.f, sched, stats, init_dev);
        MB_CUDA(cudaMemcpyAsync(rank_out, pr.rank.p, bytes, cudaMemcpyDefault, ctx->c.stream));
        MB_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

}  // extern "C"
