// learn.cu -- the learned superstep scheduler: timing traces, training, inference.
//
// Traces.  For a seeded graph and source, a base run gives the supersteps'
// features and choices: the fixed rule, or the learned policy itself when
// it is the context's policy (so a second pass of traces covers the states
// the learned policy reaches, which fixed-rule runs never visit).  Then, for every superstep i and every
// schedule s, the run is replayed with the fixed choices before i and s at
// i, and superstep i is timed alone (CUDA events around its branch in the
// host-driven loop).  The state before superstep i is the same in every
// replay (every schedule computes identical results), so the eight times
// compare the schedules on one frontier.  One sample = (features of i, eight
// costs), the cost of s being the time of superstep i under s plus the next
// kHorizon supersteps under the fixed rule.
//
// Training.  FP32 MLP 6 -> 32 -> 32 -> 8 (ReLU), hand-written kernels:
// per-sample forward and backward with gradients summed per CTA in shared
// memory, then Adam.  The target of a sample is a cost-sensitive softmax
// over its schedules' times: q_s ~ exp(-(t_s - t_min) / (tau * t_min)),
// loss = sum over samples of w_i * cross-entropy(q_i, softmax(out_i)) with
// w_i = t_min,i / sum_j t_min,j: a superstep weighs as much as the time it
// takes at best, so the fit favours the supersteps that dominate a run.
//
// Inference runs in the one-warp select kernel between supersteps
// (mlp_pick_warp in sched.cuh); k_pick exposes the same function for checks.
#include <algorithm>
#include <cmath>
#include "bfs.cuh"
#include "sssp.cuh"
#include "msbfs.cuh"
#include "learn.cuh"

namespace mb {
namespace {

constexpr int kTrainThreads = 128;
constexpr float kTau = 0.25f;  // target temperature, relative to the best time
constexpr size_t kTraceSteps = 64;  // samples per traced traversal, at most
// A schedule's cost at superstep i is the time of supersteps i .. i+kHorizon
// with that schedule at i and the fixed rule after it: the choice also sets
// the frontier format (and size) the next supersteps start from.
constexpr int32_t kHorizon = 3;

struct GradArgs {
    const float *X;  // [n][kFeat]
    const float *T;  // [n][kOut] times (ms); <= 0 or non-finite: not measured
    int32_t n;
    const float *P;  // parameters
    float *G;        // gradient (weighted mean over samples), zeroed by the caller
    float *loss;     // [0] weighted mean loss, zeroed by the caller; [1] sum of t_min
};

__device__ __forceinline__ float best_time(const float *t) {
    float tmin = 3.0e38f;
    for (int s = 0; s < kOut; s++)
        if (t[s] > 0.f && t[s] < tmin) tmin = t[s];
    return tmin;
}

// sum over samples of their best measured time (samples with none: 0)
__global__ void k_weight_sum(const float *T, int32_t n, float *out) {
    float acc = 0.f;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float tm = best_time(&T[(size_t)i * kOut]);
        if (tm < 3.0e38f) acc += tm;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0 && acc != 0.f) atomicAdd(out, acc);
}

__device__ __forceinline__ float target(const float *t, float *q) {
    const float tmin = best_time(t);
    float z = 0.f;
    for (int s = 0; s < kOut; s++) {
        q[s] = (t[s] > 0.f && t[s] < 3.0e38f) ? expf(-(t[s] - tmin) / (kTau * tmin)) : 0.f;
        z += q[s];
    }
    for (int s = 0; s < kOut; s++) q[s] = z > 0.f ? q[s] / z : 0.f;
    return z > 0.f ? tmin : 0.f;
}

__global__ void __launch_bounds__(kTrainThreads) k_mlp_grad(GradArgs a) {
    __shared__ float sg[kMlpParams];
    __shared__ float sl;
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) sg[i] = 0.f;
    if (threadIdx.x == 0) sl = 0.f;
    __syncthreads();
    const float *P = a.P;
    const float wsum = a.loss[1];
    const float inv_w = wsum > 0.f ? 1.0f / wsum : 0.f;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        float x[kFeat], z1[kHid], h1[kHid], z2[kHid], h2[kHid], o[kOut], p[kOut], q[kOut];
        for (int f = 0; f < kFeat; f++) x[f] = a.X[(size_t)i * kFeat + f];
        for (int j = 0; j < kHid; j++) {
            float acc = P[MlpLayout::b1 + j];
            for (int f = 0; f < kFeat; f++) acc = fmaf(P[MlpLayout::w1 + j * kFeat + f], x[f], acc);
            z1[j] = acc;
            h1[j] = fmaxf(acc, 0.f);
        }
        for (int k = 0; k < kHid; k++) {
            float acc = P[MlpLayout::b2 + k];
            for (int j = 0; j < kHid; j++) acc = fmaf(P[MlpLayout::w2 + k * kHid + j], h1[j], acc);
            z2[k] = acc;
            h2[k] = fmaxf(acc, 0.f);
        }
        float omax = -3.0e38f;
        for (int s = 0; s < kOut; s++) {
            float acc = P[MlpLayout::b3 + s];
            for (int k = 0; k < kHid; k++) acc = fmaf(P[MlpLayout::w3 + s * kHid + k], h2[k], acc);
            o[s] = acc;
            omax = fmaxf(omax, acc);
        }
        float z = 0.f;
        for (int s = 0; s < kOut; s++) {
            p[s] = expf(o[s] - omax);
            z += p[s];
        }
        const float wi = target(&a.T[(size_t)i * kOut], q) * inv_w;
        float l = 0.f;
        for (int s = 0; s < kOut; s++) {
            p[s] /= z;
            if (q[s] > 0.f) l -= q[s] * logf(fmaxf(p[s], 1e-30f));
        }
        atomicAdd(&sl, l * wi);
        // backward: d out = p - q
        float dz2[kHid];
        for (int k = 0; k < kHid; k++) dz2[k] = 0.f;
        for (int s = 0; s < kOut; s++) {
            const float d = (p[s] - q[s]) * wi;
            atomicAdd(&sg[MlpLayout::b3 + s], d);
            for (int k = 0; k < kHid; k++) {
                atomicAdd(&sg[MlpLayout::w3 + s * kHid + k], d * h2[k]);
                dz2[k] = fmaf(P[MlpLayout::w3 + s * kHid + k], d, dz2[k]);
            }
        }
        float dz1[kHid];
        for (int j = 0; j < kHid; j++) dz1[j] = 0.f;
        for (int k = 0; k < kHid; k++) {
            const float d = z2[k] > 0.f ? dz2[k] : 0.f;
            atomicAdd(&sg[MlpLayout::b2 + k], d);
            for (int j = 0; j < kHid; j++) {
                atomicAdd(&sg[MlpLayout::w2 + k * kHid + j], d * h1[j]);
                dz1[j] = fmaf(P[MlpLayout::w2 + k * kHid + j], d, dz1[j]);
            }
        }
        for (int j = 0; j < kHid; j++) {
            const float d = z1[j] > 0.f ? dz1[j] : 0.f;
            atomicAdd(&sg[MlpLayout::b1 + j], d);
            for (int f = 0; f < kFeat; f++) atomicAdd(&sg[MlpLayout::w1 + j * kFeat + f], d * x[f]);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x)
        if (sg[i] != 0.f) atomicAdd(&a.G[i], sg[i]);
    if (threadIdx.x == 0) atomicAdd(a.loss, sl);
}

__global__ void k_adam(float *P, const float *G, float *m, float *v, int t, float lr, float wd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float g = G[i];
    m[i] = b1 * m[i] + (1.f - b1) * g;
    v[i] = b2 * v[i] + (1.f - b2) * g * g;
    const float mh = m[i] / (1.f - powf(b1, (float)t));
    const float vh = v[i] / (1.f - powf(b2, (float)t));
    P[i] -= lr * (mh / (sqrtf(vh) + eps) + wd * P[i]);
}

// Per-feature range of the training set into P[kBoundsOff ..]: lo then hi
// (features are >= 0, so their bit patterns order like the values).
__global__ void k_feat_bounds(const float *X, int32_t n, float *P) {
    unsigned *lo = (unsigned *)&P[kBoundsOff], *hi = (unsigned *)&P[kBoundsOff + kFeat];
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int f = 0; f < kFeat; f++) {
            const unsigned b = __float_as_uint(fmaxf(X[(size_t)i * kFeat + f], 0.f));
            atomicMin(&lo[f], b);
            atomicMax(&hi[f], b);
        }
}

__global__ void k_bounds_init(float *P, float lo, float hi) {
    if (threadIdx.x < kFeat) {
        P[kBoundsOff + threadIdx.x] = lo;
        P[kBoundsOff + kFeat + threadIdx.x] = hi;
    }
}

// He-uniform initialisation from a seeded hash (deterministic)
__global__ void k_mlp_init(float *P, uint64_t seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    float fan_in = 0.f;
    if (i < MlpLayout::b1) fan_in = kFeat;
    else if (i >= MlpLayout::w2 && i < MlpLayout::b2) fan_in = kHid;
    else if (i >= MlpLayout::w3 && i < MlpLayout::b3) fan_in = kHid;
    if (fan_in == 0.f) {
        P[i] = 0.f;  // biases
        return;
    }
    const float r = (float)(hash2(seed, (uint64_t)i) >> 40) / (float)(1ull << 24);  // [0,1)
    const float lim = sqrtf(6.f / fan_in);
    P[i] = (2.f * r - 1.f) * lim;
}

__global__ void k_pick(const float *P, const float *X, const int32_t *fallback, int32_t n,
                       int32_t *out) {
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        float f[kFeat];
        for (int k = 0; k < kFeat; k++) f[k] = X[i * kFeat + k];
        MlpRegs r;
        mlp_load_warp(P, r);
        const int s = fallback ? mlp_decide_warp(r, f, 0xffu, fallback[i], kOverrideMargin)
                               : mlp_decide_warp(r, f, 0xffu, -1, 0.f);
        if ((threadIdx.x & 31) == 0) out[i] = s;
    }
}

}  // namespace

void mlp_grad(Context &ctx, const float *P_dev, const float *X_dev, const float *T_dev, int32_t n,
              float *G_dev, float *loss_dev) {
    cudaStream_t s = ctx.stream;
    MB_CUDA(cudaMemsetAsync(G_dev, 0, sizeof(float) * kMlpParams, s));
    MB_CUDA(cudaMemsetAsync(loss_dev, 0, 2 * sizeof(float), s));
    k_weight_sum<<<std::max(1, std::min(ctx.num_sms, (n + 255) / 256)), 256, 0, s>>>(T_dev, n,
                                                                                  loss_dev + 1);
    GradArgs a{X_dev, T_dev, n, P_dev, G_dev, loss_dev};
    const int grid = std::max(1, std::min(ctx.num_sms * 2, (n + kTrainThreads - 1) / kTrainThreads));
    k_mlp_grad<<<grid, kTrainThreads, 0, s>>>(a);
    MB_CHECK_LAUNCH();
}

float mlp_train(Context &ctx, float *P, const float *X_dev, const float *T_dev, int32_t n,
                int32_t epochs, float lr, uint64_t seed) {
    cudaStream_t s = ctx.stream;
    DevBuf G, M, Vb, L;
    G.reserve(sizeof(float) * kMlpParams);
    M.reserve(sizeof(float) * kMlpParams);
    Vb.reserve(sizeof(float) * kMlpParams);
    L.reserve(2 * sizeof(float));
    const int pb = (kMlpParams + 255) / 256;
    k_mlp_init<<<pb, 256, 0, s>>>(P, seed);
    MB_CUDA(cudaMemsetAsync(M.p, 0, sizeof(float) * kMlpParams, s));
    MB_CUDA(cudaMemsetAsync(Vb.p, 0, sizeof(float) * kMlpParams, s));
    for (int t = 1; t <= epochs; t++) {
        mlp_grad(ctx, P, X_dev, T_dev, n, G.as<float>(), L.as<float>());
        k_adam<<<pb, 256, 0, s>>>(P, G.as<float>(), M.as<float>(), Vb.as<float>(), t, lr, 1e-4f);
        MB_CHECK_LAUNCH();
    }
    mlp_grad(ctx, P, X_dev, T_dev, n, G.as<float>(), L.as<float>());
    k_bounds_init<<<1, 32, 0, s>>>(P, 3.0e38f, 0.f);
    k_feat_bounds<<<std::max(1, std::min(ctx.num_sms, (n + 255) / 256)), 256, 0, s>>>(X_dev, n, P);
    MB_CHECK_LAUNCH();
    float loss = 0.f;
    MB_CUDA(cudaMemcpyAsync(&loss, L.p, sizeof(float), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    G.release(); M.release(); Vb.release(); L.release();
    return loss;
}

void mlp_set_open_bounds(Context &ctx, float *P) {
    k_bounds_init<<<1, 32, 0, ctx.stream>>>(P, -3.0e38f, 3.0e38f);
    MB_CHECK_LAUNCH();
}

void mlp_pick(Context &ctx, const float *P, const float *X_dev, const int32_t *fallback_dev,
              int32_t n, int32_t *out_dev) {
    if (n <= 0) return;
    k_pick<<<std::min(ctx.num_sms * 8, (n + 7) / 8), 256, 0, ctx.stream>>>(P, X_dev, fallback_dev,
                                                                           n, out_dev);
    MB_CHECK_LAUNCH();
}

int32_t collect_traces(Context &ctx, Graph &g, BfsState &bst, SsspState &sst, MsBfsState &mst,
                       int app, int32_t source, float *feat_out, float *times_out,
                       int32_t *fixed_out, int32_t max_samples) {
    // the settings a traced replay needs; restored on return
    const int policy = ctx.schedule_policy, fixed = ctx.fixed_schedule, max_step = ctx.max_step;
    const float delta = ctx.sssp_delta;
    const bool graphs = ctx.use_graphs, tail = ctx.tail, persist = ctx.persist,
               tracing = ctx.tracing, rtf = ctx.replay_then_fixed;
    const std::vector<int8_t> replay = ctx.replay;
    // the traces are of BSP supersteps: the asynchronous SSSP kernel (which
    // runs a whole traversal as one superstep) stays off while collecting
    const int64_t async = ctx.tunable[MB_TUNE_SSSP_ASYNC];
    ctx.tunable[MB_TUNE_SSSP_ASYNC] = 0;
    auto restore = [&] {
        ctx.tunable[MB_TUNE_SSSP_ASYNC] = async;
        ctx.schedule_policy = policy;
        ctx.fixed_schedule = fixed;
        ctx.max_step = max_step;
        ctx.use_graphs = graphs;
        ctx.tail = tail;
        ctx.persist = persist;
        ctx.tracing = tracing;
        ctx.replay_then_fixed = rtf;
        ctx.replay = replay;
        ctx.sssp_delta = delta;
        ctx.trace.clear();
    };
    // batched BFS: sources `source` and the 63 vertices after it (mod V)
    const int32_t nms = (int32_t)std::min<int64_t>(64, g.V);
    std::vector<int32_t> ms_src(nms);
    for (int32_t i = 0; i < nms; i++) ms_src[i] = (int32_t)(((int64_t)source + i) % g.V);
    int32_t *ms_out = nullptr;
    if (app == APP_MSBFS) {
        mst.ensure(g);
        ms_out = (int32_t *)mst.out.reserve(sizeof(int32_t) * (size_t)nms * g.V);
    }
    auto run = [&] {
        ctx.trace.clear();
        if (app == APP_BFS) run_bfs(ctx, g, bst, source, nullptr);
        else if (app == APP_SSSP) run_sssp(ctx, g, sst, source, nullptr);
        else run_msbfs(ctx, g, mst, ms_src.data(), nms, ms_out, nullptr);
    };
    int32_t n = 0;
    try {
        // the tail stays as configured: it is what small frontiers run on
        // under schedule 0, and a trace record then spans its supersteps
        ctx.use_graphs = false;
        ctx.persist = false;
        ctx.tracing = true;
        ctx.max_step = -1;
        ctx.sssp_delta = 0.f;  // superstep i of every replay is the same superstep
        ctx.schedule_policy = policy == MB_POLICY_LEARNED ? MB_POLICY_LEARNED : MB_POLICY_FIXED;
        run();
        const std::vector<Context::TraceRec> base = ctx.trace;
        // the base run's schedule per superstep (a tail record covers the
        // supersteps up to the next record)
        std::vector<int8_t> seq;
        for (size_t k = 0; k < base.size(); k++) {
            const int32_t end = k + 1 < base.size() ? base[k + 1].step : base[k].step + 1;
            for (int32_t t = base[k].step; t < end; t++) {
                if ((int32_t)seq.size() <= t) seq.resize((size_t)t + 1, (int8_t)base[k].sched);
                seq[t] = (int8_t)base[k].sched;
            }
        }
        ctx.schedule_policy = MB_POLICY_ORACLE_BEST;
        ctx.replay_then_fixed = true;
        // a long traversal is sampled at kTraceSteps evenly spaced supersteps
        // (each sample replays its prefix: cost grows with the step index)
        const size_t stride = std::max<size_t>(1, (base.size() + kTraceSteps - 1) / kTraceSteps);
        for (size_t i = 0; i < base.size() && n < max_samples; i += stride) {
            if (base[i].sched >= MB_NUM_SCHEDULES) continue;  // internal steps (splits)
            const int32_t step = base[i].step;
            float t[MB_NUM_SCHEDULES];
            for (int sch = 0; sch < MB_NUM_SCHEDULES; sch++) {
                t[sch] = -1.f;
                // the batched traversal has two directions: push (0) and pull (4)
                if (app == APP_MSBFS && sch != MB_SCHED_PUSH_EDGE_QUEUE && sch != MB_SCHED_PULL_THREAD)
                    continue;
                ctx.replay.assign(seq.begin(), seq.begin() + std::min<size_t>(seq.size(), step));
                ctx.replay.push_back((int8_t)sch);
                ctx.max_step = step + kHorizon;
                run();
                bool ran = false;
                float sum = 0.f;
                for (const auto &r : ctx.trace) {
                    if (r.step == step) ran = true;
                    if (r.step >= step && r.step <= step + kHorizon) sum += r.ms;
                }
                if (ran) t[sch] = sum;
            }
            for (int f = 0; f < kFeat; f++) feat_out[(size_t)n * kFeat + f] = base[i].feat[f];
            for (int sch = 0; sch < MB_NUM_SCHEDULES; sch++) times_out[(size_t)n * kOut + sch] = t[sch];
            if (fixed_out) fixed_out[n] = base[i].sched;
            n++;
        }
    } catch (...) {
        restore();
        throw;
    }
    restore();
    return n;
}

}  // namespace mb
