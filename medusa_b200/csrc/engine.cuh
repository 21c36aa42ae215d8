// engine.cuh -- the frontier-driven BSP superstep engine shared by the BFS
// and SSSP apps: control block, per-superstep decision, loop-graph select
// kernel, and queue <-> bitmap frontier conversions.
//
// A superstep of either app runs one of MB_NUM_SCHEDULES schedules (see
// include/medusa_b200.h).  Schedules 0-1 read a queue frontier, 2-5 a bitmap
// frontier, 6-7 need neither; 0-1 leave a queue, all others a bitmap.  When
// the next schedule needs the other format, its loop-graph branch first runs
// a conversion (branch = schedule + MB_NUM_SCHEDULES).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include "frontier.cuh"
#include "loopgraph.cuh"
#include "sched.cuh"

namespace mb {

constexpr int FMT_QUEUE = 0, FMT_BITMAP = 1, FMT_NONE = 2;
constexpr int ERR_STEP_CAP = 1;
constexpr int kMaxReplay = 4096;
constexpr int APP_BFS = 0, APP_SSSP = 1;

// Per-run parameters, written by the host before each run (one small copy),
// so an instantiated loop graph serves every source and policy.
struct RunParams {
    int32_t source;
    int32_t policy;
    int32_t forced;
    int32_t nreplay;
    uint32_t launches;          // kernels launched by this run (device-counted)
    int8_t replay[kMaxReplay];  // MB_POLICY_ORACLE_BEST: schedule per superstep
};

// Device-resident control block of one run.
struct Ctrl {
    RunParams p;
    unsigned long long q[2];  // queue counters, packed (count << 32 | edge sum)
    int32_t cur;              // queue holding the current frontier
    int32_t bcur;             // bitmap holding the current frontier
    int32_t step;             // superstep number (BFS: level of the frontier)
    int32_t mode;             // FMT_QUEUE or FMT_BITMAP
    int32_t sched;            // schedule of the next superstep
    int32_t branch;           // loop-graph branch of the next superstep
    int32_t done;
    int32_t err;
    int32_t iter;
    int32_t supersteps;
    uint32_t blocks_done;     // last-CTA detection
    uint32_t nf;              // frontier size when in a bitmap
    uint64_t mf;              // frontier out-edges when in a bitmap
    uint32_t acc_n;           // accumulators of the running superstep
    uint64_t acc_m;
    uint32_t prev_nf;
    uint32_t front_n;
    uint64_t front_m;
    int64_t m_unvisited;      // BFS: out-edges of unvisited vertices
    int64_t n_unvisited;
    float skew;               // log2(max out-degree / mean)
    float feat[8];
    int32_t sched_count[MB_NUM_SCHEDULES];
    uint64_t reached, edges_reached;
};

// Frontier buffers and graph shape every engine kernel sees.
struct FrontierArgs {
    int32_t V;
    int64_t E;
    int64_t W;  // bitmap words
    const int32_t *outdeg;
    uint32_t *bm[2];
    int32_t *qv[2];
    uint32_t *qo[2];
    int32_t *tf[2];
    Ctrl *ctrl;
    const float *mlp;  // scheduler weights (kMlpParams floats) or null
};

__host__ __device__ inline int sched_input(int s) {
    return s <= 1 ? FMT_QUEUE : (s <= 5 ? FMT_BITMAP : FMT_NONE);
}
__host__ __device__ inline int sched_output(int s) { return s <= 1 ? FMT_QUEUE : FMT_BITMAP; }
__host__ __device__ inline int branch_of(int s, int mode) {
    const int in = sched_input(s);
    return s + ((in != FMT_NONE && in != mode) ? MB_NUM_SCHEDULES : 0);
}

// ---- the fixed rule ----------------------------------------------------------
// BFS: direction-optimising (Beamer, Asanovic & Patterson, SC 2012) -- go
// bottom-up when the frontier's out-edges exceed the unvisited out-edges /
// alpha, come back top-down when the frontier shrinks below V / beta.
// SSSP: pull (a full min over in-edges) once the frontier's out-edges are a
// large share of E, push otherwise.
__device__ inline int fixed_rule(const Ctrl *c, int app, int32_t V, int64_t E, uint32_t n,
                                 uint64_t m) {
    if (app == APP_SSSP) return (int64_t)m * 3 > E ? MB_SCHED_PULL_THREAD : MB_SCHED_PUSH_EDGE_QUEUE;
    const int64_t alpha = 15, beta = 20;
    if (c->mode == FMT_QUEUE) {
        if ((int64_t)m * alpha > c->m_unvisited) return MB_SCHED_PULL_THREAD;
        return MB_SCHED_PUSH_EDGE_QUEUE;
    }
    if ((int64_t)n * beta < (int64_t)V && n < c->prev_nf) return MB_SCHED_PUSH_EDGE_QUEUE;
    return MB_SCHED_PULL_THREAD;
}

// Decide the next superstep from the current frontier (one thread).
__device__ inline void choose_next(Ctrl *c, int app, int32_t V, int64_t E) {
    uint32_t n;
    uint64_t m;
    if (c->mode == FMT_QUEUE) {
        n = (uint32_t)(c->q[c->cur] >> 32);
        m = (uint32_t)c->q[c->cur];
    } else {
        n = c->nf;
        m = c->mf;
    }
    c->front_n = n;
    c->front_m = m;
    if (n == 0 || m == 0) {  // nothing left to expand
        c->done = 1;
        return;
    }
    int s;
    switch (c->p.policy) {
        case MB_POLICY_FORCED: s = c->p.forced; break;
        case MB_POLICY_ORACLE_BEST:
            s = c->step < c->p.nreplay ? c->p.replay[c->step] : c->p.forced;
            break;
        default: s = fixed_rule(c, app, V, E, n, m); break;
    }
    // features for the learned scheduler (the select kernel runs the MLP)
    make_features(c->feat, (double)n, (double)m, (double)c->n_unvisited, (double)c->m_unvisited,
                  (double)V, (double)E, (double)c->skew, c->mode);
    if (s < 0 || s >= MB_NUM_SCHEDULES) s = 0;
    c->sched = s;
    c->branch = branch_of(s, c->mode);
}

// Called by thread 0 of the last CTA of a superstep kernel.
__device__ inline void finish_superstep(Ctrl *c, int app, int32_t V, int64_t E, int out_fmt) {
    c->sched_count[c->sched]++;
    c->supersteps++;
    if (out_fmt == FMT_QUEUE) {
        c->cur ^= 1;
        c->q[c->cur ^ 1] = 0ull;
        c->mode = FMT_QUEUE;
        c->m_unvisited -= (int64_t)(uint32_t)c->q[c->cur];
        c->n_unvisited -= (int64_t)c->acc_n;  // every claimed vertex, queued or not
        c->acc_n = 0;
        c->acc_m = 0;
        c->prev_nf = (uint32_t)(c->q[c->cur] >> 32);
    } else {
        c->bcur ^= 1;
        c->mode = FMT_BITMAP;
        c->q[0] = 0ull;  // bitmap mode: both queues empty (k_bm2q fills q[cur])
        c->q[1] = 0ull;
        c->nf = c->acc_n;
        c->mf = c->acc_m;
        c->acc_n = 0;
        c->acc_m = 0;
        c->m_unvisited -= (int64_t)c->mf;
        c->n_unvisited -= (int64_t)c->nf;
    }
    c->step++;
    const uint32_t prev = c->prev_nf;
    choose_next(c, app, V, E);
    if (out_fmt != FMT_QUEUE) c->prev_nf = c->nf;
    (void)prev;
}

// Every engine kernel counts itself once (block 0, thread 0).
__device__ __forceinline__ void count_launch(Ctrl *c) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&c->p.launches, 1u);
}

// Last-CTA detection; true in thread 0 of the last CTA to finish.
__device__ __forceinline__ bool last_block(Ctrl *c) {
    __shared__ bool is_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned t = atomicAdd(&c->blocks_done, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        __threadfence();
        c->blocks_done = 0;
        return true;
    }
    return false;
}

// Warp-level accumulation of (new frontier vertices, their out-edges).
__device__ __forceinline__ void flush_counts(Ctrl *c, uint32_t n, uint64_t m) {
    n = warp_sum(n);
    m = warp_sum(m);
    if ((threadIdx.x & 31) == 0 && (n | m)) {
        atomicAdd(&c->acc_n, n);
        atomicAdd((unsigned long long *)&c->acc_m, (unsigned long long)m);
    }
}

__device__ __forceinline__ uint32_t warp_incl_scan_u32(uint32_t x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Warp-wide gather over the concatenated edge lists of the 32 lanes: lane L
// owns `cnt` edges starting at CSR position `start`; `incl` is the inclusive
// warp prefix of cnt.  f(valid, e) is called by all lanes, 32 edges at a time.
template <class F>
__device__ __forceinline__ void warp_gather(uint32_t incl, uint32_t cnt, int32_t start, F &&f) {
    const int lane = threadIdx.x & 31;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t k = base + lane;
        int lo = 0, hi = 31;  // first lane whose inclusive prefix exceeds k
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            const uint32_t pm = __shfl_sync(0xffffffffu, incl, mid);
            if (pm > k) hi = mid; else lo = mid + 1;
        }
        const uint32_t pinc = __shfl_sync(0xffffffffu, incl, lo);
        const uint32_t pcnt = __shfl_sync(0xffffffffu, cnt, lo);
        const int32_t pst = __shfl_sync(0xffffffffu, start, lo);
        const bool valid = k < total;
        f(valid, valid ? pst + (int32_t)(k - (pinc - pcnt)) : 0, lo);
    }
}

__device__ __forceinline__ uint32_t tail_mask(int64_t w, int32_t V) {
    return (w * 32 + 32 <= V) ? 0xffffffffu : ((1u << (uint32_t)(V - w * 32)) - 1u);
}

// ---- kernels shared by the apps (internal linkage: one copy per app file) --

// Top of every loop iteration (one warp): stop the loop when done or past
// the superstep cap; otherwise, under the learned policy, run the MLP on the
// features the last superstep left; then pick the branch.
static __global__ void k_select(Ctrl *c, const float *mlp, int cap,
                                cudaGraphConditionalHandle h_cont,
                                cudaGraphConditionalHandle h_branch, int nbranch,
                                int use_handles) {
    count_launch(c);
    const bool learned = c->p.policy == MB_POLICY_LEARNED && !c->done && mlp;
    if (learned) {  // warp-uniform
        float f[kFeat];
#pragma unroll
        for (int i = 0; i < kFeat; i++) f[i] = c->feat[i];
        const int s = mlp_pick_warp(mlp, f, 0xffu);
        if (threadIdx.x == 0) {
            c->sched = s;
            c->branch = branch_of(s, c->mode);
        }
        __syncwarp();
    }
    if (threadIdx.x != 0) return;
    c->iter++;
    if (c->iter > cap && !c->done) {
        c->err |= ERR_STEP_CAP;
        c->done = 1;
    }
    if (!use_handles) return;
    if (c->done) {
        cudaGraphSetConditional(h_branch, (unsigned)nbranch);  // no branch
        cudaGraphSetConditional(h_cont, 0);
    } else {
        cudaGraphSetConditional(h_branch, (unsigned)c->branch);
    }
}

// Zero a bitmap picked at run time: which = 0 current, 1 next.
static __global__ void k_bm_clear(FrontierArgs a, int which) {
    count_launch(a.ctrl);
    uint32_t *bm = a.bm[a.ctrl->bcur ^ which];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.W;
         i += (int64_t)gridDim.x * blockDim.x)
        bm[i] = 0u;
}

// queue q[cur] -> bitmap bm[bcur] (cleared before)
static __global__ void k_q2bm(FrontierArgs a) {
    count_launch(a.ctrl);
    Ctrl *c = a.ctrl;
    const uint32_t n = (uint32_t)(c->q[c->cur] >> 32);
    const int32_t *qv = a.qv[c->cur];
    uint32_t *bm = a.bm[c->bcur];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = qv[i];
        atomicOr(&bm[v >> 5], 1u << (v & 31));
    }
    if (last_block(c)) {
        c->nf = n;
        c->mf = (uint32_t)c->q[c->cur];
        c->q[c->cur] = 0ull;  // both queues empty in bitmap mode
        c->mode = FMT_BITMAP;
    }
}

// bitmap bm[bcur] -> queue q[cur] (empty); one warp per word
static __global__ void k_bm2q(FrontierArgs a) {
    count_launch(a.ctrl);
    Ctrl *c = a.ctrl;
    const uint32_t *bm = a.bm[c->bcur];
    const int cur = c->cur;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.W; w += warps) {
        const uint32_t word = bm[w];
        if (!word) continue;  // warp-uniform
        const int32_t v = (int32_t)(w * 32 + lane);
        const bool in = (word >> lane) & 1u;
        const uint32_t deg = in ? (uint32_t)a.outdeg[v] : 0u;
        enqueue_warp(in && deg > 0, v, deg, &c->q[cur], a.qv[cur], a.qo[cur], a.tf[cur]);
    }
    if (last_block(c)) c->mode = FMT_QUEUE;
}

// ---- host side ------------------------------------------------------------------

struct Context;

// Frontier buffers of one app on one graph, plus its instantiated loop graph.
struct FrontierState {
    bool built = false;
    int32_t V = 0;
    int64_t E = 0, W = 0;
    const void *owner = nullptr;      // context the loop graph was built for
    const void *owner_mlp = nullptr;  // scheduler weights it was built with
    DevBuf bm[2], qv[2], qo[2], tf[2], ctrl;
    LoopGraph lg;
    void release_frontier() {
        lg.reset();
        for (int i = 0; i < 2; i++) {
            bm[i].release();
            qv[i].release();
            qo[i].release();
            tf[i].release();
        }
        ctrl.release();
        owner = owner_mlp = nullptr;
        built = false;
    }
    // returns true when (re)allocated
    bool ensure_frontier(const Graph &g) {
        if (built && V == g.V && E == g.E) return false;
        release_frontier();
        V = g.V;
        E = g.E;
        W = (V + 31) / 32;
        const size_t tiles = (size_t)(E / kTile) + 2;
        for (int i = 0; i < 2; i++) {
            bm[i].reserve(sizeof(uint32_t) * (size_t)W);
            qv[i].reserve(sizeof(int32_t) * (size_t)V);
            qo[i].reserve(sizeof(uint32_t) * (size_t)V);
            tf[i].reserve(sizeof(int32_t) * tiles);
        }
        ctrl.reserve(sizeof(Ctrl));
        MB_CUDA(cudaMemset(ctrl.p, 0, sizeof(Ctrl)));
        MB_CUDA(cudaMemset(bm[0].p, 0, sizeof(uint32_t) * (size_t)W));
        MB_CUDA(cudaMemset(bm[1].p, 0, sizeof(uint32_t) * (size_t)W));
        float skew = 0.f;
        if (g.E > 0 && g.V > 0) {
            const double mean = (double)g.E / (double)g.V;
            skew = (float)std::log2(std::max(1.0, (double)g.max_outdeg / mean));
        }
        MB_CUDA(cudaMemcpy(&ctrl.as<Ctrl>()->skew, &skew, sizeof(float), cudaMemcpyHostToDevice));
        built = true;
        return true;
    }
    FrontierArgs frontier_args(const Graph &g, const float *mlp) const {
        FrontierArgs a;
        a.V = g.V;
        a.E = g.E;
        a.W = W;
        a.outdeg = g.outdeg.as<int32_t>();
        for (int i = 0; i < 2; i++) {
            a.bm[i] = bm[i].as<uint32_t>();
            a.qv[i] = qv[i].as<int32_t>();
            a.qo[i] = qo[i].as<uint32_t>();
            a.tf[i] = tf[i].as<int32_t>();
        }
        a.ctrl = ctrl.as<Ctrl>();
        a.mlp = mlp;
        return a;
    }
};

// Write this run's RunParams (policy, forced schedule, replay list, source)
// to the control block (RunParams is its first member).
void upload_params(Context &ctx, void *ctrl_dev, int32_t source);

// Run a loop (graph mode or host-driven mode) and time it; fills the common
// part of stats from the control block.
struct LoopSpec {
    FrontierState *st;
    FrontierArgs fa;
    int cap;
    EmitFn prologue;
    EmitBranch branch;
    EmitFn epilogue;
    const char *name;
};
void run_loop(Context &ctx, LoopSpec &spec, mb_stats *stats);

}  // namespace mb
