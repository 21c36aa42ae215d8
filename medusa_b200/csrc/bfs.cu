// bfs.cu -- the BFS app's BSP superstep on sm_100a.
//
// Reference semantics (Algorithm/UserOperators.h:17-35 applied to every edge
// by edgeProcWrapper, MedusaRT/APIKernelWrappers.h:35-44, once per superstep;
// CPU form Algorithm/CPUFunctorHoster.cpp:16-65): in superstep s every edge
// (u,v) with level[u] == s and level[v] == -1 sets level[v] = s+1; the loop
// stops after a superstep that set nothing.  The result is the BFS level of
// every vertex (-1 unreached) and does not depend on which edges a superstep
// looks at, so each superstep may run any of these schedules:
//
//   0 push, merge-path edge-balanced, queue frontier
//   1 push, warp-per-vertex (small lists gathered warp-wide), queue frontier
//   2 push, warp-wide edge-balanced over a bitmap frontier
//   3 push, warp-per-vertex over a bitmap frontier
//   4 pull, thread-per-vertex with a warp-cooperative tail, bitmap frontier
//   5 pull, warp-per-vertex, bitmap frontier
//   6 the reference's own form: a sweep over all E edges testing level[u]==s
//   7 pull over all vertices testing level[u]==s (no frontier structure)
//
// Every schedule writes the same levels; they differ only in the memory
// they touch.  The choice is made on the device at the end of each superstep
// (fixed rule, forced id, or the learned scheduler), so whole traversals run
// as one CUDA graph launch with no host round trip per superstep.
#include "bfs.cuh"

namespace mb {
namespace {

struct BfsArgs {
    FrontierArgs f;
    const int32_t *row, *col, *esrc, *rrow, *rcol;
    int32_t *level;
    uint32_t *vis;
};

// Claim v for level s+1.  Returns true for exactly one caller per vertex.
__device__ __forceinline__ bool claim(const BfsArgs &a, int32_t v) {
    const uint32_t bit = 1u << (v & 31);
    if (a.vis[v >> 5] & bit) return false;
    return !(atomicOr(&a.vis[v >> 5], bit) & bit);
}

// ---------------------------------------------------------------------------
// kernels

// schedule 0: push, merge-path edge-balanced over the queue
struct PushSmem {
    uint32_t off[kTile + 1];
    int32_t row[kTile + 1];
    BlockQueue bq;
};

__device__ __forceinline__ void work_push_edge_q(const BfsArgs &a, PushSmem &sm) {
    uint32_t *s_off = sm.off;
    int32_t *s_row = sm.row;
    BlockQueue &bq = sm.bq;
    if (threadIdx.x == 0) bq.n = 0;
    __syncthreads();
    Ctrl *c = a.f.ctrl;
    const int cur = c->cur, nxt = cur ^ 1;
    const uint64_t q = c->q[cur];
    const uint32_t n = (uint32_t)(q >> 32), m = (uint32_t)q;
    const int32_t lvl = c->step + 1;
    const int32_t *qv = pick(a.f.qv, cur);
    const uint32_t *qo = pick(a.f.qo, cur);
    const int32_t *tf = pick(a.f.tf, cur);
    const uint32_t tiles = (m + kTile - 1) / kTile;
    uint32_t cn = 0;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t c0 = t * kTile, c1 = min(c0 + kTile, m);
        const int32_t i0 = tf[t];
        const int32_t i1 = (t + 1 < tiles) ? tf[t + 1] : (int32_t)n - 1;
        const int k = i1 - i0 + 1;
        for (int j = threadIdx.x; j < k; j += blockDim.x) {
            s_off[j] = qo[i0 + j];
            s_row[j] = a.row[qv[i0 + j]];
        }
        __syncthreads();
        // the thread's kTileItems CONSECUTIVE edges: one binary search for the
        // first, then walk; all loads first, then the claims
        int32_t v[kTileItems];
        uint32_t vw[kTileItems];
        bool ok[kTileItems];
        {
            const uint32_t e0 = c0 + threadIdx.x * kTileItems;
            int j = e0 < c1 ? upper_bound_minus1(s_off, k, e0) : 0;
#pragma unroll
            for (int r = 0; r < kTileItems; r++) {
                const uint32_t e_idx = e0 + r;
                ok[r] = e_idx < c1;
                v[r] = 0;
                if (ok[r]) {
                    while (j + 1 < k && s_off[j + 1] <= e_idx) j++;
                    v[r] = __ldg(&a.col[s_row[j] + (int32_t)(e_idx - s_off[j])]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kTileItems; r++) vw[r] = ok[r] ? a.vis[v[r] >> 5] : ~0u;
#pragma unroll
        for (int r = 0; r < kTileItems; r++) {
            bool own = false;
            uint32_t deg = 0;
            const uint32_t bit = 1u << (v[r] & 31);
            if (ok[r] && !(vw[r] & bit) && !(atomicOr(&a.vis[v[r] >> 5], bit) & bit)) {
                own = true;
                a.level[v[r]] = lvl;
                deg = (uint32_t)a.f.outdeg[v[r]];
                cn++;
            }
            bq_push(bq, own && deg > 0, v[r], deg);
        }
        bq_flush(bq, &c->q[nxt], pick(a.f.qv, nxt), pick(a.f.qo, nxt), pick(a.f.tf, nxt));
    }
    flush_counts(c, cn, 0);
}

__global__ void __launch_bounds__(kPushThreads) k_push_edge_q(BfsArgs a) {
    __shared__ PushSmem sm;
    count_launch(a.f.ctrl);
    work_push_edge_q(a, sm);
}

// schedule 1: push, warp-per-vertex for lists >= 32, warp-wide gather below
__global__ void __launch_bounds__(kPushThreads) k_push_warp_q(BfsArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const int cur = c->cur, nxt = cur ^ 1;
    const uint32_t n = (uint32_t)(c->q[cur] >> 32);
    const int32_t lvl = c->step + 1;
    const int32_t *qv = pick(a.f.qv, cur);
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    auto visit = [&](bool valid, int32_t e) {
        bool own = false;
        int32_t v = 0;
        uint32_t deg = 0;
        if (valid) {
            v = a.col[e];
            if (claim(a, v)) {
                own = true;
                a.level[v] = lvl;
                deg = (uint32_t)a.f.outdeg[v];
                cn++;
            }
        }
        enqueue_warp(own && deg > 0, v, deg, &c->q[nxt], pick(a.f.qv, nxt), pick(a.f.qo, nxt), pick(a.f.tf, nxt));
    };
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < n;
         base += warps * 32) {
        const int64_t i = base + lane;
        int32_t u = 0, st = 0;
        uint32_t deg = 0;
        if (i < n) {
            u = qv[i];
            st = a.row[u];
            deg = (uint32_t)a.f.outdeg[u];
        }
        // large lists: whole warp, one list at a time
        unsigned big = __ballot_sync(0xffffffffu, deg >= 32);
        while (big) {
            const int l = __ffs(big) - 1;
            big &= big - 1;
            const int32_t bst = __shfl_sync(0xffffffffu, st, l);
            const uint32_t bdeg = __shfl_sync(0xffffffffu, deg, l);
            for (uint32_t k = 0; k < bdeg; k += 32) visit(k + lane < bdeg, bst + (int32_t)(k + lane));
        }
        // small lists: warp-wide gather
        const uint32_t sd = deg < 32 ? deg : 0u;
        const uint32_t incl = warp_incl_scan_u32(sd);
        warp_gather(incl, sd, st, [&](bool valid, int32_t e, int) { visit(valid, e); });
    }
    flush_counts(c, cn, 0);
}

// Discovery with a bitmap output: claim, level, next bit, counters.
__device__ __forceinline__ void discover_bm(const BfsArgs &a, uint32_t *next, int32_t v, int32_t lvl,
                                            uint32_t &cn, uint64_t &cm) {
    if (claim(a, v)) {
        a.level[v] = lvl;
        atomicOr(&next[v >> 5], 1u << (v & 31));
        cn++;
        cm += (uint32_t)a.f.outdeg[v];
    }
}

// schedules 2 and 3: push over a bitmap frontier; one warp per word.
template <bool kEdgeBalanced>
__global__ void __launch_bounds__(kPushThreads) k_push_bm(BfsArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const uint32_t *front = pick(a.f.bm, c->bcur);
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t lvl = c->step + 1;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    uint64_t cm = 0;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.f.W; w += warps) {
        const uint32_t word = front[w];
        if (!word) continue;
        const int32_t u = (int32_t)(w * 32 + lane);
        const bool in = (word >> lane) & 1u;
        const int32_t st = in ? a.row[u] : 0;
        const uint32_t deg = in ? (uint32_t)a.f.outdeg[u] : 0u;
        if (kEdgeBalanced) {
            const uint32_t incl = warp_incl_scan_u32(deg);
            warp_gather(incl, deg, st, [&](bool valid, int32_t e, int) {
                if (valid) discover_bm(a, next, a.col[e], lvl, cn, cm);
            });
        } else {
            unsigned live = __ballot_sync(0xffffffffu, deg > 0);
            while (live) {
                const int l = __ffs(live) - 1;
                live &= live - 1;
                const int32_t bst = __shfl_sync(0xffffffffu, st, l);
                const uint32_t bdeg = __shfl_sync(0xffffffffu, deg, l);
                for (uint32_t k = lane; k < bdeg; k += 32)
                    discover_bm(a, next, a.col[bst + (int32_t)k], lvl, cn, cm);
            }
        }
    }
    flush_counts(c, cn, cm);
}

constexpr int kPullLaneCap = 32;  // in-edges a lane scans alone before the warp helps

// schedule 4: pull, thread-per-vertex with a warp-cooperative tail.
// Each warp owns one word of the output bitmap and of vis.
__device__ __forceinline__ void work_pull_thread(const BfsArgs &a) {
    Ctrl *c = a.f.ctrl;
    const uint32_t *front = pick(a.f.bm, c->bcur);
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t lvl = c->step + 1;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    uint64_t cm = 0;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.f.W; w += warps) {
        const uint32_t visw = a.vis[w];
        const int32_t v = (int32_t)(w * 32 + lane);
        const uint32_t valid = tail_mask(w, a.f.V);
        const uint32_t todo = ~visw & valid;
        if (!todo) {
            if (lane == 0) next[w] = 0u;
            continue;
        }
        bool found = false;
        int32_t j = 0, je = 0;
        if ((todo >> lane) & 1u) {
            j = a.rrow[v];
            je = a.rrow[v + 1];
            const int32_t jcap = min(je, j + kPullLaneCap);
            for (; j < jcap; j++) {
                if (test_bit(front, a.rcol[j])) {
                    found = true;
                    break;
                }
            }
            if (found) je = j;  // nothing left
        }
        // lanes with long unfinished lists: the warp scans them together
        unsigned pend = __ballot_sync(0xffffffffu, !found && j < je);
        while (pend) {
            const int l = __ffs(pend) - 1;
            pend &= pend - 1;
            const int32_t pj = __shfl_sync(0xffffffffu, j, l);
            const int32_t pje = __shfl_sync(0xffffffffu, je, l);
            bool hit = false;
            for (int32_t b = pj; b < pje; b += 32) {
                const int32_t jj = b + lane;
                const bool h = jj < pje && test_bit(front, a.rcol[jj]);
                if (__any_sync(0xffffffffu, h)) {
                    hit = true;
                    break;
                }
            }
            if (lane == l) found = hit;
        }
        const uint32_t mask = __ballot_sync(0xffffffffu, found);
        if (lane == 0) {
            next[w] = mask;
            a.vis[w] = visw | mask;
        }
        if (found) {
            a.level[v] = lvl;
            cn++;
            cm += (uint32_t)a.f.outdeg[v];
        }
    }
    flush_counts(c, cn, cm);
}

__global__ void __launch_bounds__(256) k_pull_thread(BfsArgs a) {
    count_launch(a.f.ctrl);
    work_pull_thread(a);
}

// schedule 5: pull, warp-per-vertex
__global__ void __launch_bounds__(256) k_pull_warp(BfsArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const uint32_t *front = pick(a.f.bm, c->bcur);
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t lvl = c->step + 1;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    uint64_t cm = 0;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.f.W; w += warps) {
        const uint32_t visw = a.vis[w];
        const uint32_t valid = tail_mask(w, a.f.V);
        uint32_t todo = ~visw & valid;
        uint32_t mask = 0;
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const int32_t v = (int32_t)(w * 32 + l);
            const int32_t jb = a.rrow[v], je = a.rrow[v + 1];
            for (int32_t b = jb; b < je; b += 32) {
                const int32_t jj = b + lane;
                const bool h = jj < je && test_bit(front, a.rcol[jj]);
                if (__any_sync(0xffffffffu, h)) {
                    mask |= 1u << l;
                    break;
                }
            }
        }
        if (lane == 0) {
            next[w] = mask;
            a.vis[w] = visw | mask;
        }
        if ((mask >> lane) & 1u) {
            const int32_t v = (int32_t)(w * 32 + lane);
            a.level[v] = lvl;
            cn++;
            cm += (uint32_t)a.f.outdeg[v];
        }
    }
    flush_counts(c, cn, cm);
}

// schedule 6: the reference's edge-centric superstep over all E edges
// (UpdateLevel, Algorithm/UserOperators.h:17-35), next frontier as a bitmap.
__global__ void __launch_bounds__(256) k_edge_sweep(BfsArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t s = c->step;
    uint32_t cn = 0;
    uint64_t cm = 0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < a.f.E;
         e += (int64_t)gridDim.x * blockDim.x) {
        if (a.level[a.esrc[e]] == s) {
            const int32_t v = a.col[e];
            if (a.level[v] == -1) discover_bm(a, next, v, s + 1, cn, cm);
        }
    }
    flush_counts(c, cn, cm);
}

// schedule 7: pull over all unvisited vertices testing level[u] == s.
__global__ void __launch_bounds__(256) k_pull_level(BfsArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t s = c->step;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    uint64_t cm = 0;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.f.W; w += warps) {
        const int32_t v = (int32_t)(w * 32 + lane);
        bool found = false;
        if (v < a.f.V && a.level[v] == -1) {
            for (int32_t j = a.rrow[v]; j < a.rrow[v + 1]; j++)
                if (a.level[a.rcol[j]] == s) {
                    found = true;
                    break;
                }
        }
        const uint32_t mask = __ballot_sync(0xffffffffu, found);
        if (lane == 0) {
            next[w] = mask;
            a.vis[w] |= mask;
        }
        if (found) {
            a.level[v] = s + 1;
            cn++;
            cm += (uint32_t)a.f.outdeg[v];
        }
    }
    flush_counts(c, cn, cm);
}

// reached vertices and their out-edges (the reference's traversal count)
__global__ void k_stats(BfsArgs a) {
    count_launch(a.f.ctrl);
    uint32_t n = 0;
    uint64_t m = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < a.f.V;
         v += (int64_t)gridDim.x * blockDim.x) {
        if (a.level[v] >= 0) {
            n++;
            m += (uint32_t)a.f.outdeg[v];
        }
    }
    n = warp_sum(n);
    m = warp_sum(m);
    if ((threadIdx.x & 31) == 0 && (n | m)) {
        atomicAdd((unsigned long long *)&a.f.ctrl->reached, (unsigned long long)n);
        atomicAdd((unsigned long long *)&a.f.ctrl->edges_reached, (unsigned long long)m);
    }
}

// Persistent small-frontier tail (schedule 0 in one CTA): consecutive
// supersteps in one launch while the queue frontier stays within the tail
// limits; the CTA does each superstep's bookkeeping itself.
__global__ void __launch_bounds__(kTailThreads) k_tail(BfsArgs a, int cap) {
    count_launch(a.f.ctrl);
    __shared__ uint32_t s_off[kTailEntries];
    __shared__ int32_t s_row[kTailEntries];
    __shared__ int s_go;
    __shared__ Ctrl s_ctrl;  // shadow of the control block (plain loads only)
    Ctrl *const gc = a.f.ctrl;
    ctrl_shadow_in(&s_ctrl, gc);
    Ctrl *c = &s_ctrl;
    for (;;) {
        const int cur = c->cur, nxt = cur ^ 1;
        const unsigned long long q = c->q[cur];
        const uint32_t n = (uint32_t)(q >> 32), m = (uint32_t)q;
        const int32_t lvl = c->step + 1;
        const int32_t *qv = pick(a.f.qv, cur);
        const uint32_t *qo = pick(a.f.qo, cur);
        for (uint32_t j = threadIdx.x; j < n; j += kTailThreads) {
            s_off[j] = qo[j];
            s_row[j] = a.row[qv[j]];
        }
        __syncthreads();
        uint32_t cn = 0;
        for (uint32_t base = 0; base < m; base += kTailThreads) {
            const uint32_t e_idx = base + threadIdx.x;
            bool own = false;
            int32_t v = 0;
            uint32_t deg = 0;
            if (e_idx < m) {
                const int j = upper_bound_minus1(s_off, (int)n, e_idx);
                v = __ldg(&a.col[s_row[j] + (int32_t)(e_idx - s_off[j])]);
                if (claim(a, v)) {
                    own = true;
                    a.level[v] = lvl;
                    deg = (uint32_t)a.f.outdeg[v];
                    cn++;
                }
            }
            enqueue_warp(own && deg > 0, v, deg, &c->q[nxt], pick(a.f.qv, nxt), pick(a.f.qo, nxt),
                         pick(a.f.tf, nxt));
        }
        flush_counts(c, cn, 0);
        __syncthreads();
        if (threadIdx.x == 0) {
            finish_superstep<false>(c, APP_BFS, a.f.V, a.f.E, FMT_QUEUE);
            c->iter++;
            if (c->iter > cap && !c->done) {
                c->err |= ERR_STEP_CAP;
                c->done = 1;
            }
            s_go = !c->done && c->branch == kBranchTail;
        }
        __syncthreads();
        if (!s_go) break;
    }
    if (threadIdx.x == 0) c->pending = 0;
    ctrl_shadow_out(gc, c);
}

// Persistent BSP kernel (cooperative launch, all blocks resident): runs
// consecutive supersteps of schedules 0 and 4, with their frontier
// conversions, separated by grid barriers; block 0 does each superstep's
// bookkeeping between two barriers.  Leaves when the next superstep needs
// another schedule, the run is done, or a barrier gives up.
__global__ void __launch_bounds__(kPushThreads) k_persist(BfsArgs a, int cap) {
    __shared__ PushSmem sm;
    Ctrl *c = a.f.ctrl;
    count_launch(c);
    for (;;) {
        const int s = ldg2(&c->sched), mode = ldg2(&c->mode);
        if (!persist_convert(a.f, s, mode)) break;
        if (s == MB_SCHED_PULL_THREAD) work_pull_thread(a);
        else work_push_edge_q(a, sm);
        if (!grid_sync(c)) break;
        persist_bookkeep(a.f, APP_BFS, cap);
        if (!grid_sync(c)) break;
        if (!ldg2(&c->persist_go)) break;
    }
}

__global__ void k_bfs_init(BfsArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const int32_t source = c->p.source;
    const int32_t deg = a.f.outdeg[source];
    if (threadIdx.x == 0) {
        a.level[source] = 0;
        a.vis[source >> 5] |= 1u << (source & 31);
        c->cur = 0;
        c->bcur = 0;
        c->step = 0;
        c->mode = FMT_QUEUE;
        c->done = 0;
        c->err = 0;
        c->iter = 0;
        c->supersteps = 0;
        for (int i = 0; i < MB_NUM_SCHEDULES; i++) c->sched_count[i] = 0;
        c->acc_n = 0;
        c->acc_m = 0;
        c->blocks_done = 0;
        c->prev_nf = 1;
        c->reached = 1;
        c->edges_reached = (uint64_t)deg;
        c->work = 0;
        c->pending = 0;
        c->bar_count = 0;
        c->q[1] = 0ull;
        c->m_unvisited = a.f.E - deg;
        c->n_unvisited = a.f.V - 1;
        if (deg > 0) {
            pick(a.f.qv, 0)[0] = source;
            pick(a.f.qo, 0)[0] = 0;
            c->q[0] = (1ull << 32) | (uint32_t)deg;
        } else {
            c->q[0] = 0ull;
        }
    }
    for (int32_t t = threadIdx.x; deg > 0 && t * kTile < deg; t += blockDim.x) pick(a.f.tf, 0)[t] = 0;
    __syncthreads();
    if (threadIdx.x == 0) choose_next(c, APP_BFS, a.f.V, a.f.E);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side

void run_bfs(Context &ctx, Graph &g, BfsState &st, int32_t source, mb_stats *stats, int phase, int force,
             int *cont, const EmitFn *after) {
    st.ensure(g);
    BfsArgs a;
    a.f = st.frontier_args(g, ctx.model(MB_MODEL_BFS));
    a.row = g.row.as<int32_t>();
    a.col = g.col.as<int32_t>();
    a.esrc = g.esrc.as<int32_t>();
    a.rrow = g.rrow.as<int32_t>();
    a.rcol = g.rcol.as<int32_t>();
    a.level = st.level.as<int32_t>();
    a.vis = st.vis.as<uint32_t>();
    if (phase == LOOP_ALL) upload_params(ctx, st.ctrl.p, source);
    if (phase == LOOP_BEGIN) {  // a stepped run: one superstep per call (no persistent kernels)
        const bool tail = ctx.tail, persist = ctx.persist;
        ctx.tail = ctx.persist = false;
        upload_params(ctx, st.ctrl.p, source);
        ctx.tail = tail;
        ctx.persist = persist;
    }

    const int grid_push = ctx.num_sms * ctx.blocks_per_sm(MB_TUNE_PUSH_BLOCKS_PER_SM, 8);
    const int grid_vtx = ctx.num_sms * ctx.blocks_per_sm(MB_TUNE_VERTEX_BLOCKS_PER_SM, 8);
    const int grid_edge = grid_vtx;
    const int persist_grid = persistent_grid_size(ctx, (const void *)k_persist, kPushThreads);
    LoopSpec sp;
    sp.st = &st;
    sp.fa = a.f;
    sp.app = APP_BFS;
    sp.cap = step_cap(ctx, (int64_t)g.V + 4);
    sp.name = "bfs";
    sp.prologue = [&](cudaStream_t s) {
        MB_CUDA(cudaMemsetAsync(a.level, 0xff, sizeof(int32_t) * (size_t)a.f.V, s));
        MB_CUDA(cudaMemsetAsync(a.vis, 0, sizeof(uint32_t) * (size_t)a.f.W, s));
        k_bfs_init<<<1, 256, 0, s>>>(a);
        MB_CHECK_LAUNCH();
    };
    sp.branch = [&](int branch, cudaStream_t s) {
        // BFS never routes to the bitmap-output push (bm_push_min is 0) nor
        // to the asynchronous kernel (sssp_async is 0)
        if (branch == kBranchPushBm || branch == kBranchAsync) branch = MB_SCHED_PUSH_EDGE_QUEUE;
        if (branch == kBranchPushSmall) {
            k_push_edge_q<<<ctx.num_sms * kSmallPushPerSm, kPushThreads, 0, s>>>(a);
            MB_CHECK_LAUNCH();
            return;
        }
        if (branch == kBranchTail) {
            k_tail<<<1, kTailThreads, 0, s>>>(a, sp.cap);
            MB_CHECK_LAUNCH();
            return;
        }
        if (branch == kBranchPersist) {
            launch_cooperative((const void *)k_persist, persist_grid, kPushThreads, s, a, sp.cap);
            return;
        }
        const int sched = branch % MB_NUM_SCHEDULES;
        if (branch >= MB_NUM_SCHEDULES) {
            if (sched_input(sched) == FMT_BITMAP) {
                k_bm_clear<<<grid_vtx, 256, 0, s>>>(a.f, 0);
                k_q2bm<<<grid_vtx, 256, 0, s>>>(a.f);
            } else {
                k_bm2q<<<grid_vtx, 256, 0, s>>>(a.f);
            }
            MB_CHECK_LAUNCH();
        }
        switch (sched) {
            case MB_SCHED_PUSH_EDGE_QUEUE: k_push_edge_q<<<grid_push, kPushThreads, 0, s>>>(a); break;
            case MB_SCHED_PUSH_WARP_QUEUE: k_push_warp_q<<<grid_push, kPushThreads, 0, s>>>(a); break;
            case MB_SCHED_PUSH_EDGE_BITMAP:
                k_bm_clear<<<grid_vtx, 256, 0, s>>>(a.f, 1);
                k_push_bm<true><<<grid_push, kPushThreads, 0, s>>>(a);
                break;
            case MB_SCHED_PUSH_WARP_BITMAP:
                k_bm_clear<<<grid_vtx, 256, 0, s>>>(a.f, 1);
                k_push_bm<false><<<grid_push, kPushThreads, 0, s>>>(a);
                break;
            case MB_SCHED_PULL_THREAD: k_pull_thread<<<grid_vtx, 256, 0, s>>>(a); break;
            case MB_SCHED_PULL_WARP: k_pull_warp<<<grid_vtx, 256, 0, s>>>(a); break;
            case MB_SCHED_PUSH_UNFUSED:
                k_bm_clear<<<grid_vtx, 256, 0, s>>>(a.f, 1);
                k_edge_sweep<<<grid_edge, 256, 0, s>>>(a);
                break;
            default: k_pull_level<<<grid_vtx, 256, 0, s>>>(a); break;
        }
        MB_CHECK_LAUNCH();
    };
    sp.epilogue = nullptr;  // reached counts are kept by finish_superstep
    if (after) sp.after = *after;
    run_loop(ctx, sp, stats, phase, force, cont);
}

}  // namespace mb
