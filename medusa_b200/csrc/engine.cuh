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
#include "runparams.cuh"
#include "sched.cuh"

namespace mb {

constexpr int FMT_QUEUE = 0, FMT_BITMAP = 1, FMT_NONE = 2;
constexpr int ERR_STEP_CAP = 1;
constexpr int ERR_BARRIER = 2;     // a grid barrier of the persistent kernel gave up
constexpr int ERR_BULK = 4;        // a bulk copy into shared memory did not complete in time
constexpr int ERR_ASYNC = 8;       // a wait of the asynchronous SSSP kernel gave up
// Internal step of near-far SSSP (not a user schedule): raise the distance
// threshold and move far-pile vertices below it into the near queue.
constexpr int kSchedSplit = MB_NUM_SCHEDULES;
constexpr int kBranchSplit = 2 * MB_NUM_SCHEDULES;
// Persistent small-frontier tail: schedule 0 run by ONE CTA of kTailThreads
// threads for as many consecutive supersteps as the frontier stays within
// kTailEntries vertices and kTailEdges edges (no launch per superstep).
constexpr int kBranchTail = kBranchSplit + 1;
// Persistent BSP kernel: one cooperative grid runs consecutive supersteps of
// schedules 0 and 4 (with their frontier conversions) and near-far splits,
// separated by grid barriers, until a superstep needs anything else.
constexpr int kBranchPersist = kBranchTail + 1;
// Schedule 0 of SSSP on a large queue frontier: the relaxations set bits of
// a next-frontier bitmap with fire-and-forget atomics (no per-vertex claim
// round trip), and a compaction pass turns the bitmap into the next queue.
constexpr int kBranchPushBm = kBranchPersist + 1;
// Schedule 0 on a medium queue frontier (above the tail's limits, at most
// p.small_push_max out-edges): the same push on a grid of two CTAs per SM,
// which dispatches and retires faster than the full grid.
constexpr int kBranchPushSmall = kBranchPushBm + 1;
// SSSP schedule 0 on a queue frontier with asynchronous relaxation on: one
// cooperative launch relaxes until no distance can drop (the rest of the
// traversal, without superstep barriers).
constexpr int kBranchAsync = kBranchPushSmall + 1;
constexpr int kNumBranches = kBranchAsync + 1;
constexpr int kSmallPushPerSm = 2;  // CTAs per SM of the small-grid push
constexpr int kTailThreads = 1024;
constexpr uint32_t kTailEntries = 2048, kTailEdges = 8192;
// The SSSP tail keeps its frontier in shared memory: room for kSTailCap
// next-frontier vertices (<= the frontier's out-edges, <= kTailEdges) and a
// hash set of twice that.
constexpr int kSTailCap = 8192;
constexpr size_t kTailSmemBytes = 4 * (size_t)(2 * kSTailCap + 3 * kSTailCap + kTailEntries + 33);
static_assert(kTailEdges <= (uint32_t)kSTailCap, "tail edges exceed the shared-memory tail");

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
    uint64_t work;            // edges examined: push frontier out-edges, E per pull/sweep
    int32_t pending;          // a superstep ran and awaits finish_superstep
    float thresh;             // SSSP near-far: vertices below go to the near queue
    uint32_t far_n[2];        // SSSP near-far: far-pile sizes
    int32_t fcur;             // far pile being filled
    int32_t splits;           // near-far split steps run
    uint32_t bar_count;       // persistent-grid barrier: arrivals over the run (top bit: gave up)
    uint32_t pad_bar;
    int32_t persist_go;       // persistent grid: run another superstep
    int32_t peaked;           // SSSP: a frontier reached p.async_below out-edges
    uint32_t far_min;         // SSSP near-far: float bits of the least distance the last split kept (+inf: none)
    float thresh_prev;        // SSSP near-far: the threshold before the last raise
    int32_t pad_far;
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
__host__ __device__ inline int sched_output(int s) {
    return (s <= 1 || s == kSchedSplit) ? FMT_QUEUE : FMT_BITMAP;
}
__host__ __device__ inline int branch_of(int s, int mode) {
    if (s == kSchedSplit) return kBranchSplit;
    const int in = sched_input(s);
    return s + ((in != FMT_NONE && in != mode) ? MB_NUM_SCHEDULES : 0);
}

// The branch that runs schedule s from the current frontier: the persistent
// tail for a small queue frontier under schedule 0.
__device__ inline int route(const struct Ctrl *c, int s);

// ---- the fixed rule ----------------------------------------------------------
// BFS: direction-optimising (Beamer, Asanovic & Patterson, SC 2012) -- go
// bottom-up when the frontier's out-edges exceed the unvisited out-edges /
// alpha, come back top-down when the frontier shrinks below V / beta.
// SSSP: always push, edge-balanced.  An SSSP pull must scan every in-edge to
// find what a push reaches through the frontier's out-edges, and a minimum
// has no early exit, so pulling never does less work.
__device__ inline int fixed_rule(const Ctrl *c, int app, int32_t V, int64_t E, uint32_t n,
                                 uint64_t m) {
    if (app == APP_SSSP) return MB_SCHED_PUSH_EDGE_QUEUE;
    const int64_t alpha = c->p.bfs_alpha, beta = c->p.bfs_beta;  // default 15 and 20
    const int64_t gamma = c->p.bfs_gamma;
    if (c->mode == FMT_QUEUE) {
        // bottom-up only for a frontier that is large in absolute terms too
        // (at least E / gamma out-edges): near the end of a high-diameter
        // traversal the unvisited out-edges run low while the frontier stays
        // small, and a pull over every unvisited vertex costs more than the push
        if (alpha > 0 && (int64_t)m * alpha > c->m_unvisited && (gamma == 0 || (int64_t)m * gamma >= E))
            return MB_SCHED_PULL_THREAD;
        return MB_SCHED_PUSH_EDGE_QUEUE;
    }
    if ((int64_t)n * beta < (int64_t)V && n < c->prev_nf) return MB_SCHED_PUSH_EDGE_QUEUE;
    return MB_SCHED_PULL_THREAD;
}

__host__ __device__ inline bool persist_supported(int s) {
    return s == MB_SCHED_PUSH_EDGE_QUEUE || s == MB_SCHED_PULL_THREAD || s == kSchedSplit;
}

__device__ inline int route(const Ctrl *c, int s) {
    if (c->p.persist && persist_supported(s)) return kBranchPersist;
    if (s == MB_SCHED_PUSH_EDGE_QUEUE && c->mode == FMT_QUEUE && c->p.sssp_async &&
        (c->p.async_below == 0 || (c->peaked && c->front_m < c->p.async_below)))
        return kBranchAsync;
    if (s == MB_SCHED_PUSH_EDGE_QUEUE && c->mode == FMT_QUEUE && c->p.tail &&
        c->front_n <= kTailEntries && c->front_m <= c->p.tail_edges)
        return kBranchTail;
    if (s == MB_SCHED_PUSH_EDGE_QUEUE && c->mode == FMT_QUEUE && c->p.bm_push_min &&
        c->front_m >= c->p.bm_push_min)
        return kBranchPushBm;
    if (s == MB_SCHED_PUSH_EDGE_QUEUE && c->mode == FMT_QUEUE && c->front_m <= c->p.small_push_max)
        return kBranchPushSmall;
    return branch_of(s, c->mode);
}

// Counters other CTAs updated with atomics: read at L2 (kL2) where those
// CTAs may still be running (the persistent kernels), a plain load in the
// select kernel (every superstep kernel has finished; its bookkeeping reads
// the control block after one warp-wide prefetch into L1).
template <bool kL2, class T>
__device__ __forceinline__ T ctl_ld(const T *p) {
    if (kL2) return ldg2(p);
    return *p;
}

// Decide the next superstep from the current frontier (one thread).
template <bool kL2 = true>
__device__ inline void choose_next(Ctrl *c, int app, int32_t V, int64_t E) {
    uint32_t n;
    uint64_t m;
    if (c->mode == FMT_QUEUE) {
        const unsigned long long q = ctl_ld<kL2>(&c->q[c->cur]);
        n = (uint32_t)(q >> 32);
        m = (uint32_t)q;
    } else {
        n = c->nf;
        m = c->mf;
    }
    c->front_n = n;
    c->front_m = m;
    if (c->p.async_below && m >= c->p.async_below) c->peaked = 1;
    if (c->p.max_step >= 0 && c->step > c->p.max_step) {  // trace collection: stop here
        c->done = 1;
        return;
    }
    if (n == 0 || m == 0) {  // nothing left to expand
        if (app == APP_SSSP && ctl_ld<kL2>(&c->far_n[c->fcur]) > 0) {
            // near-far: next bucket.  The threshold rises by delta, and past
            // the least distance the last split kept in the far pile (empty
            // buckets are skipped: their count would not be bounded by the
            // superstep cap); one float step further where a sum rounds back.
            const float fm = __uint_as_float(ctl_ld<kL2>(&c->far_min));
            const bool known = fm < __uint_as_float(0x7f800000u);
            float t = c->thresh + c->p.delta;
            if (known) t = fmaxf(t, fm + c->p.delta);
            if (!(t > c->thresh)) t = __uint_as_float(__float_as_uint(c->thresh) + 1u);
            if (known && !(t > fm)) t = __uint_as_float(__float_as_uint(fm) + 1u);
            c->thresh_prev = c->thresh;
            c->thresh = t;
            c->far_min = 0x7f800000u;
            c->sched = kSchedSplit;
            c->branch = route(c, kSchedSplit);
            return;
        }
        c->done = 1;
        return;
    }
    int s;
    switch (c->p.policy) {
        case MB_POLICY_FORCED: s = c->p.forced; break;
        case MB_POLICY_ORACLE_BEST:
            if (c->step < c->p.nreplay) s = c->p.replay[c->step];
            else s = c->p.replay_then_fixed ? fixed_rule(c, app, V, E, n, m) : c->p.forced;
            break;
        default: s = fixed_rule(c, app, V, E, n, m); break;
    }
    // features for the learned scheduler (the select kernel runs the MLP)
    make_features(c->feat, (float)n, (float)m, (float)c->n_unvisited, (float)c->m_unvisited,
                  (float)V, (float)E, c->skew, c->mode);
    if (s < 0 || s >= MB_NUM_SCHEDULES) s = 0;
    c->sched = s;
    c->branch = route(c, s);
}

// Bookkeeping after a superstep (one thread).
template <bool kL2 = true>
__device__ inline void finish_superstep(Ctrl *c, int app, int32_t V, int64_t E, int out_fmt) {
    if (c->sched == kSchedSplit) {
        c->splits++;
        c->far_n[c->fcur] = 0;
        c->fcur ^= 1;
        c->supersteps++;
    } else {
        c->sched_count[c->sched]++;
        c->supersteps++;
        c->work += c->sched <= MB_SCHED_PUSH_WARP_BITMAP ? c->front_m : (uint64_t)E;
    }
    // accumulators and queue counters were updated with atomics
    const uint32_t acc_n = ctl_ld<kL2>(&c->acc_n);
    const uint64_t acc_m = ctl_ld<kL2>((const unsigned long long *)&c->acc_m);
    const unsigned long long qn = ctl_ld<kL2>(&c->q[c->cur ^ 1]);
    if (app == APP_BFS) {  // claimed vertices and their out-edges
        c->reached += acc_n;
        c->edges_reached += out_fmt == FMT_QUEUE ? (uint32_t)qn : acc_m;
    }
    if (out_fmt == FMT_QUEUE) {
        c->cur ^= 1;
        c->q[c->cur ^ 1] = 0ull;
        c->mode = FMT_QUEUE;
        c->m_unvisited -= (int64_t)(uint32_t)qn;
        c->n_unvisited -= (int64_t)acc_n;  // every claimed vertex, queued or not
        c->acc_n = 0;
        c->acc_m = 0;
        c->prev_nf = (uint32_t)(qn >> 32);
    } else {
        c->bcur ^= 1;
        c->mode = FMT_BITMAP;
        c->q[0] = 0ull;  // bitmap mode: both queues empty (k_bm2q fills q[cur])
        c->q[1] = 0ull;
        c->nf = acc_n;
        c->mf = acc_m;
        c->acc_n = 0;
        c->acc_m = 0;
        c->m_unvisited -= (int64_t)c->mf;
        c->n_unvisited -= (int64_t)c->nf;
    }
    c->step++;
    choose_next<kL2>(c, app, V, E);
    if (out_fmt != FMT_QUEUE) c->prev_nf = c->nf;
}

// The single-CTA tails run with a shadow of the control block in shared
// memory (no other kernel runs while a tail does): the per-superstep
// bookkeeping of thread 0 and the counter atomics of every thread then cost
// shared-memory latency, not a chain of L2 round trips.  Code given the
// shadow reads it with plain loads (ldg2 / ctl_ld<true> address global
// memory only).  Called by every thread of the CTA.
static_assert(sizeof(Ctrl) % 8 == 0, "control block copied in 8-byte words");
static_assert(offsetof(Ctrl, q) % 8 == 0, "the select kernel writes back from q on, in 8-byte words");
// The replay list (4 KB of the run parameters) is copied only for the
// replay policy, and every thread issues all of its loads before its stores:
// one L2 round trip per pass instead of one per word.
static_assert(offsetof(Ctrl, p) == 0 && offsetof(RunParams, replay) % 8 == 0 && kMaxReplay % 8 == 0,
              "the replay list is skipped in 8-byte words");
constexpr int kCtrlWords = (int)(sizeof(Ctrl) / 8);
constexpr int kReplayW0 = (int)(offsetof(RunParams, replay) / 8);
constexpr int kReplayW1 = kReplayW0 + kMaxReplay / 8;
constexpr int kHotWords = kReplayW0 + (kCtrlWords - kReplayW1);  // words outside the replay list
__device__ __forceinline__ int hot_word(int i) { return i < kReplayW0 ? i : i - kReplayW0 + kReplayW1; }
__device__ inline void ctrl_shadow_in(Ctrl *s, const Ctrl *g) {
    const auto *gw = reinterpret_cast<const unsigned long long *>(g);
    auto *sw = reinterpret_cast<unsigned long long *>(s);
    for (int base = 0; base < kHotWords; base += 4 * (int)blockDim.x) {
        unsigned long long v[4];
        int w[4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int i = base + r * (int)blockDim.x + (int)threadIdx.x;
            w[r] = i < kHotWords ? hot_word(i) : -1;
            v[r] = w[r] >= 0 ? __ldcg(&gw[w[r]]) : 0ull;
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
            if (w[r] >= 0) sw[w[r]] = v[r];
    }
    __syncthreads();
    if (s->p.policy == MB_POLICY_ORACLE_BEST) {
        for (int i = kReplayW0 + (int)threadIdx.x; i < kReplayW1; i += (int)blockDim.x) sw[i] = __ldcg(&gw[i]);
        __syncthreads();
    }
}
__device__ inline void ctrl_shadow_out(Ctrl *g, const Ctrl *s) {
    __syncthreads();
    for (int i = threadIdx.x; i < kHotWords; i += blockDim.x) {
        const int w = hot_word(i);
        reinterpret_cast<unsigned long long *>(g)[w] = reinterpret_cast<const unsigned long long *>(s)[w];
    }
    __threadfence();
}

// Every engine kernel counts itself once (block 0, thread 0).
__device__ __forceinline__ void count_launch(Ctrl *c) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&c->p.launches, 1u);
}

// Block-level accumulation of (new frontier vertices, their out-edges): one
// atomic pair per block.  Called by every thread of the block.
__device__ __forceinline__ void flush_counts(Ctrl *c, uint32_t n, uint64_t m) {
    __shared__ uint32_t s_n[32];
    __shared__ unsigned long long s_m[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    n = warp_sum(n);
    m = warp_sum(m);
    if (lane == 0) {
        s_n[wid] = n;
        s_m[wid] = m;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        uint32_t bn = lane < nw ? s_n[lane] : 0u;
        uint64_t bm = lane < nw ? s_m[lane] : 0ull;
        bn = warp_sum(bn);
        bm = warp_sum(bm);
        if (lane == 0 && (bn | bm)) {
            atomicAdd(&c->acc_n, bn);
            atomicAdd((unsigned long long *)&c->acc_m, (unsigned long long)bm);
        }
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

// One full warp: finish the superstep that ran (frontier bookkeeping and
// the choice of the next schedule), then, under the learned policy, run the
// MLP on the features it left.
template <bool kPrefetch = true>
__device__ inline void bookkeep_warp(const FrontierArgs &a, int app) {
    Ctrl *c = a.ctrl;
    if (kPrefetch) {
        // the control block's lines and the run parameters' head, all at once
        const int lane = threadIdx.x & 31;
        const char *hot = (const char *)&c->q[0];
        const size_t hot_bytes = sizeof(Ctrl) - offsetof(Ctrl, q);
        if ((size_t)lane * 128 < hot_bytes)
            asm volatile("prefetch.global.L1 [%0];" ::"l"(hot + (size_t)lane * 128));
        if (lane == 31) asm volatile("prefetch.global.L1 [%0];" ::"l"((const char *)&c->p));
        __syncwarp();
    }
    const bool use_mlp = a.mlp && c->p.policy == MB_POLICY_LEARNED;  // warp-uniform
    MlpRegs r;
    if (use_mlp) mlp_load_warp(a.mlp, r);  // in flight during the bookkeeping
    if ((threadIdx.x & 31) == 0 && c->pending) {
        c->pending = 0;
        finish_superstep<false>(c, app, a.V, a.E, sched_output(c->sched));
    }
    __syncwarp();
    const bool learned = use_mlp && !c->done && c->sched != kSchedSplit;
    if (learned) {  // warp-uniform
        float f[kFeat];
#pragma unroll
        for (int i = 0; i < kFeat; i++) f[i] = c->feat[i];
        // c->sched holds the fixed rule's choice (choose_next)
        const int s = mlp_decide_warp(r, f, 0xffu, c->sched, kOverrideMargin);
        if ((threadIdx.x & 31) == 0) {
            c->sched = s;
            c->branch = route(c, s);
        }
        __syncwarp();
    }
}

// A stepped run's next superstep with schedule s instead of the policy's.
static __global__ void k_force_sched(FrontierArgs a, int s) {
    Ctrl *c = a.ctrl;
    if (threadIdx.x == 0 && !c->done) {
        c->sched = s;
        c->branch = route(c, s);
    }
}

// Count one loop iteration; past the cap the run stops with an error, and
// so does a run in which a bounded wait gave up.
__device__ inline void count_iteration(Ctrl *c, int cap) {
    c->iter++;
    if (c->iter > cap && !c->done) {
        c->err |= ERR_STEP_CAP;
        c->done = 1;
    }
    if (c->err & (ERR_BARRIER | ERR_BULK | ERR_ASYNC)) c->done = 1;
}

// Top of every loop iteration (one warp): bookkeeping of the superstep that
// just ran (so superstep kernels need no last-CTA detection), stop the loop
// when done or past the superstep cap, else pick the branch.
static __global__ void k_select(FrontierArgs a, int app, int cap,
                                cudaGraphConditionalHandle h_cont,
                                cudaGraphConditionalHandle h_branch, int nbranch,
                                int use_handles) {
    // the warp copies the control block into shared memory (all loads in
    // flight at once), thread 0 does the bookkeeping there, and the warp
    // writes back the part after the run parameters (the only part the
    // bookkeeping changes; the launch count is added in global memory)
    Ctrl *const gc = a.ctrl;
    count_launch(gc);
    __shared__ Ctrl s_ctrl;
    ctrl_shadow_in(&s_ctrl, gc);
    FrontierArgs sa = a;
    sa.ctrl = &s_ctrl;
    bookkeep_warp<false>(sa, app);
    Ctrl *c = &s_ctrl;
    if (threadIdx.x == 0) {
        count_iteration(c, cap);
        if (!c->done) c->pending = 1;
    }
    __syncwarp();
    {
        constexpr int kFrom = (int)(offsetof(Ctrl, q) / 8), kTo = (int)(sizeof(Ctrl) / 8);
        for (int i = kFrom + (int)threadIdx.x; i < kTo; i += (int)blockDim.x)
            reinterpret_cast<unsigned long long *>(gc)[i] = reinterpret_cast<const unsigned long long *>(c)[i];
    }
    if (threadIdx.x != 0) return;
    if (!use_handles) return;
    if (c->done) {
        cudaGraphSetConditional(h_branch, (unsigned)nbranch);  // no branch
        cudaGraphSetConditional(h_cont, 0);
    } else {
        cudaGraphSetConditional(h_branch, (unsigned)c->branch);
    }
}

// Grid barrier of the persistent kernel (all blocks co-resident: cooperative
// launch).  bar_count counts arrivals over the whole run (zeroed by the
// run's init kernel), so barrier k completes when it reaches k * gridDim.x:
// one atomic per block, then polling of the same word with acquire loads
// (which also drop this SM's stale L1 lines).  The wait is bounded: past
// kBarrierSpins polls (or the run's wait_polls, when set) the block records
// ERR_BARRIER, sets the counter's top bit -- every block still waiting, and
// every later barrier, then fails at once -- and returns false, and the
// caller leaves its loop.
constexpr long kBarrierSpins = 1l << 22;
constexpr unsigned kBarPoison = 1u << 31;
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ inline bool grid_sync(Ctrl *c) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();  // this block's writes before its arrival
        const unsigned arrived = atomicAdd(&c->bar_count, 1u);
        int ok = 0;
        if (arrived < kBarPoison) {
            const unsigned target = (arrived / gridDim.x + 1) * gridDim.x;
            const long spins = c->p.wait_polls >= 0 ? (long)c->p.wait_polls : kBarrierSpins;
            for (long it = 0;; it++) {
                const unsigned v = ld_acquire_gpu(&c->bar_count);
                if (v >= kBarPoison) break;  // another block gave up
                if (v >= target) {
                    ok = 1;
                    break;
                }
                if (it >= spins) {
                    atomicOr(&c->err, ERR_BARRIER);
                    atomicOr(&c->bar_count, kBarPoison);
                    break;
                }
                __nanosleep(16);
            }
        }
        if (!ok) atomicOr(&c->err, ERR_BARRIER);
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok;
}

// The persistent kernel's bookkeeping between two barriers (block 0, warp 0):
// finish the superstep that ran and decide whether the grid runs the next one.
__device__ inline void persist_bookkeep(const FrontierArgs &a, int app, int cap) {
    Ctrl *c = a.ctrl;
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    if (threadIdx.x == 0) c->pending = 1;
    __syncwarp();
    bookkeep_warp(a, app);
    if (threadIdx.x == 0) {
        count_iteration(c, cap);
        c->persist_go = !c->done && c->branch == kBranchPersist;
        __threadfence();
    }
}

// Zero a bitmap picked at run time: which = 0 current, 1 next.
__device__ inline void work_bm_clear(const FrontierArgs &a, int which) {
    uint32_t *bm = pick(a.bm, a.ctrl->bcur ^ which);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.W;
         i += (int64_t)gridDim.x * blockDim.x)
        bm[i] = 0u;
}

// queue q[cur] -> bitmap bm[bcur] (cleared before)
__device__ inline void work_q2bm(const FrontierArgs &a) {
    Ctrl *c = a.ctrl;
    const uint32_t n = (uint32_t)(c->q[c->cur] >> 32);
    const int32_t *qv = pick(a.qv, c->cur);
    uint32_t *bm = pick(a.bm, c->bcur);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = qv[i];
        atomicOr(&bm[v >> 5], 1u << (v & 31));
    }
}

// bitmap bm[bcur] -> queue q[cur] (empty); one warp per word
__device__ inline void work_bm2q(const FrontierArgs &a) {
    Ctrl *c = a.ctrl;
    const uint32_t *bm = pick(a.bm, c->bcur);
    const int cur = c->cur;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.W; w += warps) {
        const uint32_t word = bm[w];
        if (!word) continue;  // warp-uniform
        const int32_t v = (int32_t)(w * 32 + lane);
        const bool in = (word >> lane) & 1u;
        const uint32_t deg = in ? (uint32_t)a.outdeg[v] : 0u;
        enqueue_warp(in && deg > 0, v, deg, &c->q[cur], pick(a.qv, cur), pick(a.qo, cur), pick(a.tf, cur));
    }
}

static __global__ void k_bm_clear(FrontierArgs a, int which) {
    count_launch(a.ctrl);
    work_bm_clear(a, which);
}
static __global__ void k_q2bm(FrontierArgs a) {
    count_launch(a.ctrl);
    work_q2bm(a);
}
static __global__ void k_bm2q(FrontierArgs a) {
    count_launch(a.ctrl);
    work_bm2q(a);
}

// Frontier conversion a persistent superstep of schedule s needs first
// (grid-wide, with barriers); false if a barrier gave up.
__device__ inline bool persist_convert(const FrontierArgs &a, int s, int mode) {
    const int in = sched_input(s);
    if (in == FMT_BITMAP && mode == FMT_QUEUE) {
        work_bm_clear(a, 0);
        if (!grid_sync(a.ctrl)) return false;
        work_q2bm(a);
        return grid_sync(a.ctrl);
    }
    if (in == FMT_QUEUE && mode == FMT_BITMAP) {
        work_bm2q(a);
        return grid_sync(a.ctrl);
    }
    return true;
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
    uint64_t owner_gen = ~0ull;       // tunables generation it was built with
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
            // +8: bulk copies of a tile's entries round their end up to 16 bytes
            qv[i].reserve(sizeof(int32_t) * ((size_t)V + 8));
            qo[i].reserve(sizeof(uint32_t) * ((size_t)V + 8));
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


// Run a loop (graph mode or host-driven mode) and time it; fills the common
// part of stats from the control block.
struct LoopSpec {
    FrontierState *st;
    FrontierArgs fa;
    int cap;
    int app;
    EmitFn prologue;
    EmitBranch branch;
    EmitFn epilogue;
    const char *name;
    // whole runs (LOOP_ALL): queued after the run's end event and before
    // its one host synchronisation (e.g. the copy of the run's output to the
    // caller), so that it costs no synchronisation of its own
    EmitFn after;
};
// The phases of a run driven one superstep at a time (mb_superstep): BEGIN
// runs the prologue and picks the first superstep, STEP runs the picked one
// (a schedule forced when force >= 0) and picks the next, FINISH runs the
// epilogue and reads the statistics.  ALL is a whole run (one CUDA graph
// launch, or the host-driven loop).  *cont: another superstep is needed.
enum LoopPhase { LOOP_ALL = 0, LOOP_BEGIN = 1, LOOP_STEP = 2, LOOP_FINISH = 3 };
void run_loop(Context &ctx, LoopSpec &spec, mb_stats *stats, int phase = LOOP_ALL, int force = -1,
              int *cont = nullptr);

// Blocks of the persistent kernel: every SM holds min(resident, 4) of them,
// so a cooperative launch always fits.
int persistent_grid_size(const Context &ctx, const void *kernel, int threads);

// Cooperative launch of kernel(args, cap) (capturable into a CUDA graph).
template <class Args>
void launch_cooperative(const void *kernel, int grid, int threads, cudaStream_t s, Args args,
                        int cap) {
    void *params[] = {(void *)&args, (void *)&cap};
    MB_CUDA(cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(threads), params, 0, s));
}

}  // namespace mb
