// msbfs.cu -- batched BFS: up to 64 sources in one traversal (64-bit
// per-vertex source masks).
//
// Every source s owns bit s.  seen[v] holds the sources that reached v,
// front[v] the sources whose level-L frontier contains v.  A superstep ORs
// the frontier masks across edges, so ONE scan of an edge serves every
// source whose frontier holds its tail:
//   push (sparse union frontier): for the out-edges of queued frontier
//     vertices, next[v] |= front[u] & ~seen[v]; a commit pass over the
//     touched vertices turns next into the new frontier;
//   pull (dense union frontier): each vertex still missing some sources ORs
//     the frontier masks of its in-neighbours, stopping as soon as all the
//     sources it misses are covered.
// A source's bit appears in front[v] exactly at the superstep the reference's
// single-source BFS (Algorithm/CPUFunctorHoster.cpp:16-65) would set level
// L+1, so levels_out[s*V + v] equals 64 independent runs bit for bit.  No
// reference counterpart exists for the batching itself (the reference's
// "MBFS" app is multi-GPU BFS).
//
// The loop is one CUDA graph (WHILE over a SWITCH of three branches: push,
// dense->queue + push, pull).  A one-warp select kernel at the top of each
// iteration finishes the superstep that ran and picks the direction of the
// next one: the fixed rule (pull once the union frontier's out-edges pass
// E/16), a forced or replayed schedule, or the learned scheduler's MLP
// restricted to {push, pull}.  Pull-family schedules (4, 5, 7) map to pull,
// the rest to push; every choice yields the same levels.
#include <algorithm>
#include <cmath>
#include "msbfs.cuh"
#include "sched.cuh"

namespace mb {
namespace {

struct MsCtrl {
    RunParams p;              // first member: written by upload_params
    unsigned long long q[2];  // frontier queue counters, packed (count << 32 | edges)
    uint32_t touched;         // touched vertices of a push superstep
    uint32_t active;          // frontier vertices after the superstep
    unsigned long long active_edges;
    int32_t cur;              // queue / front buffer of the current frontier
    int32_t step;
    int32_t mode;             // 0: queue frontier (push next), 1: dense (pull next)
    int32_t done;
    int32_t supersteps;
    int32_t pushes, pulls;
    int32_t pending;          // a superstep ran since the last select
    int32_t last_pull;        // its direction
    int32_t iter, err, branch, sched;
    uint32_t reached;         // vertices seen by at least one source
    unsigned long long reached_edges;  // their out-edges
    float skew;               // log2(max out-degree / mean), scheduler feature
    float feat[8];            // features of the last decision
};
constexpr int kMsBranchPush = 0, kMsBranchPull = 1, kMsBranchDensePush = 2, kMsBranches = 3;

struct MsArgs {
    int32_t V;
    int64_t E;
    const int32_t *row, *col, *rrow, *rcol, *outdeg;
    unsigned long long *seen, *front[2], *nxt;
    int32_t *touched;
    int32_t *qv[2];
    uint32_t *qo[2];
    int32_t *tf[2];
    int32_t *levels;  // [nsrc][V]
    int32_t nsrc;
    unsigned long long all;  // mask of the batch's sources
    const float *mlp;        // batched-traversal scheduler weights (nullptr: untrained)
    MsCtrl *c;
};

__device__ __forceinline__ void ms_count_launch(const MsArgs &a) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.c->p.launches, 1u);
}

__device__ __forceinline__ int32_t push_level(const MsArgs &a) { return a.c->step + 1; }

// Record the level of every source in `bits` for vertex v.
__device__ __forceinline__ void write_levels(const MsArgs &a, int32_t v, unsigned long long bits,
                                             int32_t lvl) {
    while (bits) {
        const int s = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        a.levels[(size_t)s * a.V + v] = lvl;
    }
}

__global__ void k_ms_init(MsArgs a, const int32_t *sources) {
    // one thread: sources may repeat; the queue holds each vertex once
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    MsCtrl *c = a.c;
    c->p.launches++;
    c->q[0] = c->q[1] = 0ull;
    c->cur = 0;
    c->step = 0;
    c->mode = 0;
    c->done = 0;
    c->supersteps = 0;
    c->pushes = c->pulls = 0;
    c->pending = 0;
    c->last_pull = 0;
    c->iter = 0;
    c->err = 0;
    c->branch = 0;
    c->sched = 0;
    c->touched = 0;
    uint32_t n = 0, m = 0, nr = 0;
    unsigned long long mr = 0;
    for (int i = 0; i < a.nsrc; i++) {
        const int32_t v = sources[i];
        const unsigned long long bit = 1ull << i;
        if (a.front[0][v] == 0ull) {
            const uint32_t d = (uint32_t)a.outdeg[v];
            nr++;
            mr += d;
            if (d > 0) {
                a.qv[0][n] = v;
                a.qo[0][n] = m;
                for (uint32_t t = (m + kTile - 1) / kTile; t <= (m + d - 1) / kTile; t++)
                    a.tf[0][t] = (int32_t)n;
                n++;
                m += d;
            }
        }
        a.front[0][v] |= bit;
        a.seen[v] |= bit;
        a.levels[(size_t)i * a.V + v] = 0;
    }
    c->q[0] = ((unsigned long long)n << 32) | m;
    c->active = n;
    c->active_edges = m;
    c->reached = nr;
    c->reached_edges = mr;
    c->done = n == 0;
}

struct MsPushSmem {
    uint32_t off[kTile + 1];
    int32_t row[kTile + 1];
    unsigned long long fr[kTile + 1];
};

// push: next[v] |= front[u] & ~seen[v] over the frontier queue's edges
// (merge-path tiles, one search per thread over consecutive edges)
__global__ void __launch_bounds__(kPushThreads) k_ms_push(MsArgs a) {
    __shared__ MsPushSmem sm;
    MsCtrl *c = a.c;
    ms_count_launch(a);
    const int cur = c->cur;
    const unsigned long long q = c->q[cur];
    const uint32_t n = (uint32_t)(q >> 32), m = (uint32_t)q;
    const int32_t *qv = cur ? a.qv[1] : a.qv[0];
    const uint32_t *qo = cur ? a.qo[1] : a.qo[0];
    const int32_t *tf = cur ? a.tf[1] : a.tf[0];
    const unsigned long long *front = cur ? a.front[1] : a.front[0];
    const uint32_t tiles = (m + kTile - 1) / kTile;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t c0 = t * kTile, c1 = min(c0 + kTile, m);
        const int32_t i0 = tf[t];
        const int32_t i1 = (t + 1 < tiles) ? tf[t + 1] : (int32_t)n - 1;
        const int k = i1 - i0 + 1;
        for (int j = threadIdx.x; j < k; j += blockDim.x) {
            const int32_t u = qv[i0 + j];
            sm.off[j] = qo[i0 + j];
            sm.row[j] = a.row[u];
            sm.fr[j] = front[u];
        }
        __syncthreads();
        const uint32_t e0 = c0 + threadIdx.x * kTileItems;
        int j = e0 < c1 ? upper_bound_minus1(sm.off, k, e0) : 0;
        int32_t v[kTileItems];
        unsigned long long f[kTileItems];
#pragma unroll
        for (int r = 0; r < kTileItems; r++) {
            const uint32_t e_idx = e0 + r;
            v[r] = -1;
            f[r] = 0ull;
            if (e_idx < c1) {
                while (j + 1 < k && sm.off[j + 1] <= e_idx) j++;
                v[r] = __ldg(&a.col[sm.row[j] + (int32_t)(e_idx - sm.off[j])]);
                f[r] = sm.fr[j];
            }
        }
#pragma unroll
        for (int r = 0; r < kTileItems; r++) {
            bool first = false;
            if (v[r] >= 0) {
                const unsigned long long bits = f[r] & ~__ldcg(&a.seen[v[r]]);
                if (bits) first = atomicOr(&a.nxt[v[r]], bits) == 0ull;
            }
            // warp-aggregated append of first touches
            const unsigned mask = __ballot_sync(0xffffffffu, first);
            if (mask) {
                const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(&c->touched, (uint32_t)__popc(mask));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (first) a.touched[base + __popc(mask & lanemask_lt())] = v[r];
            }
        }
        __syncthreads();
    }
}

// commit after a push: the old frontier's masks are cleared; every touched
// vertex takes its new bits (levels, seen) and joins the next queue.
__global__ void k_ms_commit(MsArgs a) {
    MsCtrl *c = a.c;
    ms_count_launch(a);
    const int cur = c->cur, nx = cur ^ 1;
    const uint32_t nold = (uint32_t)(c->q[cur] >> 32), nt = c->touched;
    unsigned long long *front_cur = cur ? a.front[1] : a.front[0];
    unsigned long long *front_nx = cur ? a.front[0] : a.front[1];
    const int32_t *qv = cur ? a.qv[1] : a.qv[0];
    const int32_t lvl = push_level(a);
    const int lane = threadIdx.x & 31;
    // grid-stride in warp-sized chunks over [0, nold + nt)
    const int64_t total = (int64_t)nold + nt;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t nr = 0;
    unsigned long long mr = 0;
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < total;
         base += warps * 32) {
        const int64_t i = base + lane;
        bool join = false;
        int32_t v = 0;
        uint32_t deg = 0;
        if (i < nold) {
            front_cur[qv[i]] = 0ull;
        } else if (i < total) {
            v = a.touched[i - nold];
            const unsigned long long old = a.seen[v];
            const unsigned long long nb = a.nxt[v] & ~old;
            a.nxt[v] = 0ull;
            if (nb) {
                if (old == 0ull) {
                    nr++;
                    mr += (uint32_t)a.outdeg[v];
                }
                a.seen[v] = old | nb;
                front_nx[v] = nb;
                write_levels(a, v, nb, lvl);
                deg = (uint32_t)a.outdeg[v];
                join = deg > 0;
            }
        }
        enqueue_warp(join, v, deg, &c->q[nx], nx ? a.qv[1] : a.qv[0], nx ? a.qo[1] : a.qo[0],
                     nx ? a.tf[1] : a.tf[0]);
    }
    nr = warp_sum(nr);
    mr = warp_sum(mr);
    if (lane == 0 && nr) {
        atomicAdd(&c->reached, nr);
        atomicAdd(&c->reached_edges, mr);
    }
}

// pull: every vertex still missing some sources ORs its in-neighbours'
// frontier masks (early exit once covered); writes the whole next buffer.
__global__ void __launch_bounds__(256) k_ms_pull(MsArgs a) {
    MsCtrl *c = a.c;
    const int cur = c->cur;
    const unsigned long long *front = cur ? a.front[1] : a.front[0];
    unsigned long long *front_nx = cur ? a.front[0] : a.front[1];
    const int32_t lvl = push_level(a);
    ms_count_launch(a);
    uint32_t act = 0, nr = 0;
    unsigned long long act_e = 0, mr = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < a.V;
         v += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long old = a.seen[v];
        const unsigned long long need = a.all & ~old;
        unsigned long long acc = 0ull;
        if (need) {
            const int32_t jb = a.rrow[v], je = a.rrow[v + 1];
            for (int32_t j = jb; j < je; j++) {
                acc |= front[__ldg(&a.rcol[j])];
                if ((acc & need) == need) break;
            }
            acc &= need;
            if (acc) {
                a.seen[v] = old | acc;
                write_levels(a, (int32_t)v, acc, lvl);
                const uint32_t d = (uint32_t)a.outdeg[v];
                if (old == 0ull) {
                    nr++;
                    mr += d;
                }
                if (d > 0) {
                    act++;
                    act_e += d;
                }
            }
        }
        front_nx[v] = acc;
    }
    act = warp_sum(act);
    act_e = warp_sum(act_e);
    nr = warp_sum(nr);
    mr = warp_sum(mr);
    if ((threadIdx.x & 31) == 0 && act) {
        atomicAdd(&c->active, act);
        atomicAdd(&c->active_edges, act_e);
    }
    if ((threadIdx.x & 31) == 0 && nr) {
        atomicAdd(&c->reached, nr);
        atomicAdd(&c->reached_edges, mr);
    }
}

// after a pull: clear the old front buffer
__global__ void k_ms_clear_front(MsArgs a) {
    ms_count_launch(a);
    unsigned long long *f = a.c->cur ? a.front[1] : a.front[0];
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < a.V;
         v += (int64_t)gridDim.x * blockDim.x)
        f[v] = 0ull;
}

// dense front -> queue of the vertices with a nonzero mask (for a push)
__global__ void k_ms_dense2q(MsArgs a) {
    MsCtrl *c = a.c;
    ms_count_launch(a);
    const int cur = c->cur;
    const unsigned long long *front = cur ? a.front[1] : a.front[0];
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < a.V;
         base += warps * 32) {
        const int64_t v = base + lane;
        uint32_t deg = 0;
        bool in = false;
        if (v < a.V && front[v]) {
            deg = (uint32_t)a.outdeg[v];
            in = deg > 0;
        }
        enqueue_warp(in, (int32_t)v, deg, &c->q[cur], cur ? a.qv[1] : a.qv[0],
                     cur ? a.qo[1] : a.qo[0], cur ? a.tf[1] : a.tf[0]);
    }
}

// superstep bookkeeping (one thread) before and after a push or a pull
__device__ void ms_begin(MsCtrl *c, int pull) {
    if (pull) {
        c->active = 0;
        c->active_edges = 0ull;
    } else {
        c->touched = 0;
        c->q[c->cur ^ 1] = 0ull;
        if (c->mode == 1) c->q[c->cur] = 0ull;  // refilled by k_ms_dense2q
    }
}

__device__ void ms_end(MsCtrl *c, int pull) {
    if (pull) {
        c->cur ^= 1;
        c->mode = 1;
        c->q[0] = c->q[1] = 0ull;
        c->pulls++;
    } else {
        const unsigned long long qn = ldg2(&c->q[c->cur ^ 1]);
        c->q[c->cur] = 0ull;
        c->cur ^= 1;
        c->mode = 0;
        c->active = (uint32_t)(qn >> 32);
        c->active_edges = (uint32_t)qn;
        c->pushes++;
    }
    c->step++;
    c->supersteps++;
    c->done = c->active == 0;
}

__device__ __forceinline__ bool pull_family(int s) {
    return s == MB_SCHED_PULL_THREAD || s == MB_SCHED_PULL_WARP || s == MB_SCHED_PULL_UNFUSED;
}

// Top of every loop iteration (one full warp): finish the superstep that
// ran, stop when done (or past the cap, or past p.max_step), else choose
// the direction of the next superstep and set the graph's conditions.
__global__ void k_ms_select(MsArgs a, int cap, cudaGraphConditionalHandle h_cont,
                            cudaGraphConditionalHandle h_branch, int use_handles) {
    MsCtrl *c = a.c;
    const int lane = threadIdx.x & 31;
    const bool use_mlp = a.mlp && c->p.policy == MB_POLICY_LEARNED;  // warp-uniform
    MlpRegs r;
    if (use_mlp) mlp_load_warp(a.mlp, r);  // in flight during the bookkeeping
    if (lane == 0) {
        c->p.launches++;
        if (c->pending) {
            c->pending = 0;
            ms_end(c, c->last_pull);
        }
        c->iter++;
        if (c->iter > cap && !c->done) {
            c->err |= 1;
            c->done = 1;
        }
        if (c->p.max_step >= 0 && c->step > c->p.max_step) c->done = 1;
    }
    __syncwarp();
    const int done = c->done;
    int s = MB_SCHED_PUSH_EDGE_QUEUE;
    if (!done) {
        const int fixed = (unsigned long long)c->active_edges * 16ull > (unsigned long long)a.E
                              ? MB_SCHED_PULL_THREAD : MB_SCHED_PUSH_EDGE_QUEUE;
        float f[kFeat];
        make_features(f, (float)c->active, (float)c->active_edges, (float)(a.V - (int64_t)c->reached),
                      (float)(a.E - (int64_t)c->reached_edges), (float)a.V, (float)a.E, c->skew,
                      c->mode);
        switch (c->p.policy) {
            case MB_POLICY_FORCED: s = c->p.forced; break;
            case MB_POLICY_ORACLE_BEST:
                if (c->step < c->p.nreplay) s = c->p.replay[c->step];
                else s = c->p.replay_then_fixed ? fixed : c->p.forced;
                break;
            case MB_POLICY_LEARNED:
                // warp-uniform: every lane runs the MLP
                s = use_mlp ? mlp_decide_warp(r, f, (1u << MB_SCHED_PUSH_EDGE_QUEUE) |
                                                        (1u << MB_SCHED_PULL_THREAD),
                                              fixed, kOverrideMargin)
                            : fixed;
                break;
            default: s = fixed; break;
        }
        if (lane < kFeat) c->feat[lane] = f[lane];
    }
    __syncwarp();
    if (lane != 0) return;
    if (done) {
        if (use_handles) {
            cudaGraphSetConditional(h_branch, (unsigned)kMsBranches);  // no branch
            cudaGraphSetConditional(h_cont, 0);
        }
        return;
    }
    const int pull = pull_family(s);
    c->sched = pull ? MB_SCHED_PULL_THREAD : MB_SCHED_PUSH_EDGE_QUEUE;
    c->branch = pull ? kMsBranchPull : (c->mode == 1 ? kMsBranchDensePush : kMsBranchPush);
    ms_begin(c, pull);
    c->last_pull = pull;
    c->pending = 1;
    if (use_handles) cudaGraphSetConditional(h_branch, (unsigned)c->branch);
}

// per-source traversal count: sum over v of popc(seen[v]) * outdeg[v]
__global__ void k_ms_stats(MsArgs a, unsigned long long *out) {
    ms_count_launch(a);
    unsigned long long er = 0, vr = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < a.V;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int p = __popcll(a.seen[v]);
        vr += p;
        er += (unsigned long long)p * (uint32_t)a.outdeg[v];
    }
    er = warp_sum(er);
    vr = warp_sum(vr);
    if ((threadIdx.x & 31) == 0 && (er | vr)) {
        atomicAdd(&out[0], er);
        atomicAdd(&out[1], vr);
    }
}

}  // namespace

void MsBfsState::ensure(const Graph &g) {
    if (built && V == g.V && E == g.E) return;
    release();
    V = g.V;
    E = g.E;
    const size_t vb = (size_t)V;
    seen.reserve(8 * vb);
    front[0].reserve(8 * vb);
    front[1].reserve(8 * vb);
    nxt.reserve(8 * vb);
    touched.reserve(4 * vb);
    const size_t tiles = (size_t)(E / kTile) + 2;
    for (int i = 0; i < 2; i++) {
        qv[i].reserve(4 * vb);
        qo[i].reserve(4 * vb);
        tf[i].reserve(4 * tiles);
    }
    ctrl.reserve(sizeof(MsCtrl));
    stats.reserve(2 * sizeof(unsigned long long));
    srcs.reserve(64 * sizeof(int32_t));
    built = true;
}

void run_msbfs(Context &ctx, Graph &g, MsBfsState &st, const int32_t *sources, int32_t nsrc,
               int32_t *levels_dev, mb_stats *stats) {
    static_assert(sizeof(MsCtrl) <= Context::kSmallBytes - Context::kCtrlOff, "ctrl readback");
    if (nsrc < 1 || nsrc > 64) fail(MB_ERR_INVALID, "batched BFS takes 1..64 sources");
    st.ensure(g);
    cudaStream_t s = ctx.stream;
    MsArgs a;
    a.V = g.V;
    a.E = g.E;
    a.row = g.row.as<int32_t>();
    a.col = g.col.as<int32_t>();
    a.rrow = g.rrow.as<int32_t>();
    a.rcol = g.rcol.as<int32_t>();
    a.outdeg = g.outdeg.as<int32_t>();
    a.seen = st.seen.as<unsigned long long>();
    a.front[0] = st.front[0].as<unsigned long long>();
    a.front[1] = st.front[1].as<unsigned long long>();
    a.nxt = st.nxt.as<unsigned long long>();
    a.touched = st.touched.as<int32_t>();
    for (int i = 0; i < 2; i++) {
        a.qv[i] = st.qv[i].as<int32_t>();
        a.qo[i] = st.qo[i].as<uint32_t>();
        a.tf[i] = st.tf[i].as<int32_t>();
    }
    a.levels = levels_dev;
    a.nsrc = nsrc;
    a.all = nsrc == 64 ? ~0ull : ((1ull << nsrc) - 1ull);
    a.mlp = ctx.model(MB_MODEL_BATCHED);
    a.c = st.ctrl.as<MsCtrl>();
    const size_t vb = (size_t)g.V;
    const int gv = ctx.num_sms * 8, gp = ctx.num_sms * 8;
    // every superstep reaches at least one new (vertex, source) pair
    const int cap = step_cap(ctx, (int64_t)g.V + 8);

    auto prologue = [&](cudaStream_t cs) {
        MB_CUDA(cudaMemsetAsync(a.seen, 0, 8 * vb, cs));
        MB_CUDA(cudaMemsetAsync(a.front[0], 0, 8 * vb, cs));
        MB_CUDA(cudaMemsetAsync(a.front[1], 0, 8 * vb, cs));
        MB_CUDA(cudaMemsetAsync(a.nxt, 0, 8 * vb, cs));
        MB_CUDA(cudaMemsetAsync(levels_dev, 0xff, sizeof(int32_t) * vb * nsrc, cs));
        MB_CUDA(cudaMemsetAsync(st.stats.p, 0, 2 * sizeof(unsigned long long), cs));
        k_ms_init<<<1, 32, 0, cs>>>(a, st.srcs.as<int32_t>());
        MB_CHECK_LAUNCH();
    };
    auto branch = [&](int b, cudaStream_t cs) {
        if (b == kMsBranchPull) {
            k_ms_pull<<<gv, 256, 0, cs>>>(a);
            k_ms_clear_front<<<gv, 256, 0, cs>>>(a);
        } else {
            if (b == kMsBranchDensePush) k_ms_dense2q<<<gv, 256, 0, cs>>>(a);
            k_ms_push<<<gp, kPushThreads, 0, cs>>>(a);
            k_ms_commit<<<gv, 256, 0, cs>>>(a);
        }
        MB_CHECK_LAUNCH();
    };
    auto epilogue = [&](cudaStream_t cs) {
        k_ms_stats<<<gv, 256, 0, cs>>>(a, st.stats.as<unsigned long long>());
        MB_CHECK_LAUNCH();
    };

    cudaEvent_t e0 = nullptr, e1 = nullptr, t0 = nullptr, t1 = nullptr;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    MsCtrl *hc = (MsCtrl *)ctx.ctrl_readback();
    auto cleanup = [&] {
        for (cudaEvent_t e : {e0, e1, t0, t1})
            if (e) cudaEventDestroy(e);
    };
    try {
        upload_params(ctx, a.c, nsrc > 0 ? sources[0] : 0);
        float skew = 0.f;
        if (g.E > 0 && g.V > 0)
            skew = (float)std::log2(std::max(1.0, (double)g.max_outdeg / ((double)g.E / g.V)));
        MB_CUDA(cudaMemcpyAsync(st.srcs.p, sources, sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
        MB_CUDA(cudaMemcpyAsync(&a.c->skew, &skew, sizeof(float), cudaMemcpyHostToDevice, s));
        const bool host_loop = !ctx.use_graphs || ctx.tracing;
        if (!host_loop && (!st.lg.exec || st.key_levels != levels_dev || st.key_nsrc != nsrc ||
                           st.key_mlp != a.mlp)) {
            build_loop_graph(
                st.lg, s, kMsBranches, prologue,
                [&](cudaStream_t cs, cudaGraphConditionalHandle hcont, cudaGraphConditionalHandle hb) {
                    k_ms_select<<<1, 32, 0, cs>>>(a, cap, hcont, hb, 1);
                    MB_CHECK_LAUNCH();
                },
                branch, epilogue);
            st.key_levels = levels_dev;
            st.key_nsrc = nsrc;
            st.key_mlp = a.mlp;
        }
        MB_CUDA(cudaEventRecord(e0, s));
        if (!host_loop) {
            MB_CUDA(cudaGraphLaunch(st.lg.exec, s));
        } else {
            prologue(s);
            if (ctx.tracing) {
                MB_CUDA(cudaEventCreate(&t0));
                MB_CUDA(cudaEventCreate(&t1));
            }
            for (;;) {
                k_ms_select<<<1, 32, 0, s>>>(a, cap, 0, 0, 0);
                MB_CHECK_LAUNCH();
                MB_CUDA(cudaMemcpyAsync(hc, a.c, sizeof(MsCtrl), cudaMemcpyDeviceToHost, s));
                MB_CUDA(cudaStreamSynchronize(s));
                if (hc->done) break;
                if (ctx.tracing) {
                    Context::TraceRec r;
                    r.app = APP_MSBFS;
                    r.step = hc->step;
                    r.sched = hc->sched;
                    r.branch = hc->branch;
                    r.n = hc->active;
                    r.m = hc->active_edges;
                    for (int i = 0; i < 8; i++) r.feat[i] = hc->feat[i];
                    MB_CUDA(cudaEventRecord(t0, s));
                    branch(hc->branch, s);
                    MB_CUDA(cudaEventRecord(t1, s));
                    MB_CUDA(cudaEventSynchronize(t1));
                    MB_CUDA(cudaEventElapsedTime(&r.ms, t0, t1));
                    ctx.trace.push_back(r);
                } else {
                    branch(hc->branch, s);
                }
            }
            epilogue(s);
        }
        MB_CUDA(cudaEventRecord(e1, s));
        MB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        MB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        MB_CUDA(cudaMemcpyAsync(hc, a.c, sizeof(MsCtrl), cudaMemcpyDeviceToHost, s));
        unsigned long long hs[2];
        MB_CUDA(cudaMemcpyAsync(hs, st.stats.p, sizeof(hs), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        if (hc->err) fail(MB_ERR_TIMEOUT, "batched bfs: superstep cap reached");
        if (stats) {
            *stats = mb_stats{};
            stats->supersteps = hc->supersteps;
            stats->edges_traversed = (int64_t)hs[0];
            stats->vertices_reached = (int64_t)hs[1];
            stats->device_ms = ms;
            stats->schedule_count[MB_SCHED_PUSH_EDGE_QUEUE] = hc->pushes;
            stats->schedule_count[MB_SCHED_PULL_THREAD] = hc->pulls;
            stats->kernel_launches = hc->p.launches;
        }
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
}

}  // namespace mb
