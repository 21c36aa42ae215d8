// sssp.cu -- the SSSP app's BSP superstep on sm_100a.
//
// Reference (SSSP/UserOperators.h:10-29,151-168,200-264; combiner
// MedusaRT/Combiner.cu:82-142 with CUDPP_MIN; CPU form
// SSSP/CPUFunctorHoster.cpp:15-99): each superstep fills an E-slot message
// array with FLT_MAX, every updated vertex writes dist[u]+w into the slot of
// each out-edge, a segmented min-scan combines the slots of each destination,
// and every vertex whose combined message is below its distance takes it and
// is "updated" for the next superstep.  The fixpoint is the exact
// shortest-path distance (1e9 = MEDUSA_MAX when unreachable): the weights are
// integers stored as float and every path length is an integer below 2^24,
// so float sums and minima are exact and the result does not depend on
// relaxation order.  Hence every schedule below yields bit-identical output.
//
// Fused schedules combine in the send: atomicMin on the float's bit pattern
// (non-negative floats order like their uint32 bits) and the "updated" set
// is the set of vertices whose distance dropped, deduplicated per superstep by
// a stamp (stamp[v] == s+1 once v joined superstep s+1's frontier).
//
//   0 push, merge-path edge-balanced, queue frontier
//   1 push, warp-per-vertex, queue frontier
//   2 push, warp-wide edge-balanced over a bitmap frontier
//   3 push, warp-per-vertex over a bitmap frontier
//   4 pull (min over in-edges from frontier vertices), edge-streamed by a
//     warp per 32 destinations
//   5 pull, warp-per-vertex
//   6 the reference's split: message fill, send into msg[mslot[e]],
//     segmented min per destination, update
//   7 full Bellman-Ford pull over every in-edge (the reference CPU form)
#include "sssp.cuh"
#include "bulk.cuh"

namespace mb {
namespace {

struct SsspArgs {
    FrontierArgs f;
    const int32_t *row, *col, *rrow, *rcol, *mslot;
    const float *wt, *rwt;
    float *dist;
    int32_t *stamp;
    float *msg;
    int32_t *far[2];  // near-far piles (vertices whose distance is >= the threshold)
    uint32_t *farbm;  // membership bitmap of the pile being filled
    uint32_t *nbm;    // next-frontier bitmap of the bitmap-output push (all zero between uses)
    float *dprev;     // distances before the superstep (the snapshot variant of that push)
    AsyncState *as;   // the asynchronous kernel's counters
    // the asynchronous kernel's dirty bitmap over vertex ids [0, V) and hub
    // chunk ids [V, V + nchunks) (a.nbm when the graph has no hub)
    uint32_t *adirty;
    int64_t WA;                   // its words
    const int32_t *hub_cbase;     // first chunk of each hub
    const int32_t *chunk_src;     // hub of the chunk at each position (id - V)
    const int32_t *chunk_rs;      // first out-edge of the chunk at each position
    int32_t nc32;                 // chunk c sits at id V + (c % 32) * nc32 + c / 32
};

__device__ __forceinline__ float ld_dist(const SsspArgs &a, int32_t v) {
    return __ldcg(&a.dist[v]);  // bypass L1: other SMs lower distances
}

// Lower dist[v] to nd; true if this call lowered it.
__device__ __forceinline__ bool lower(const SsspArgs &a, int32_t v, float nd) {
    if (!(nd < ld_dist(a, v))) return false;
    const unsigned old = atomicMin((unsigned *)&a.dist[v], __float_as_uint(nd));
    return nd < __uint_as_float(old);
}

// True for exactly one caller per (v, superstep): v joins the next frontier.
__device__ __forceinline__ bool mark(const SsspArgs &a, int32_t v, int32_t stamp_val) {
    return atomicExch(&a.stamp[v], stamp_val) != stamp_val;
}

__device__ __forceinline__ bool relax(const SsspArgs &a, int32_t v, float nd, int32_t stamp_val) {
    return lower(a, v, nd) && mark(a, v, stamp_val);
}

// Near-far: append v to the far pile being filled, once (all lanes call it).
__device__ __forceinline__ void far_push(const SsspArgs &a, Ctrl *c, bool pred, int32_t v) {
    if (pred) {
        const uint32_t bit = 1u << (v & 31);
        pred = !(atomicOr(&a.farbm[v >> 5], bit) & bit);
    }
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    const int f = c->fcur;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&c->far_n[f], (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) pick(a.far, f)[base + __popc(mask & lanemask_lt())] = v;
}

// schedule 0: push, merge-path edge-balanced over the queue
// A tile's queue entries (offsets and vertices) come into shared memory by
// the threads' own loads, or (kBulk, MB_TUNE_BULK_STAGE) by one bulk copy
// each on the TMA engine.  A tile holds at most kTile + 1 entries; the bulk
// copy rounds their range out to 16-byte boundaries (at most 3 entries on
// each side).  Measured on B200 the two are within 1% of each other.
constexpr int kStage = kTile + 8;
struct PushSmem {
    alignas(16) uint32_t qo_st[kStage];  // the offsets (threads' loads: from index 0)
    alignas(16) int32_t qv_st[kStage];   // the vertices (bulk copies only)
    uint64_t bar;
    int32_t row[kTile + 1];
    float du[kTile + 1];
    BlockQueue bq;
};

// Combining a warp's same-destination relaxations with __match_any_sync
// (one distance read and one reduction per distinct destination) measured
// 1.7x (R-MAT 2^20/2^24) to 2.4x (R-MAT 2^24/2^28) SLOWER on B200 than one
// read per edge: the match costs more than the L2 requests it saves.  Kept
// behind this switch, off.
#ifndef MB_SSSP_MATCH
#define MB_SSSP_MATCH 0
#endif
// The bitmap-output push without the per-edge distance read: every
// relaxation is a fire-and-forget atomicMin, and the next frontier is the
// set of vertices whose distance dropped below a snapshot taken before the
// superstep (plain frontier Bellman-Ford only).  Measured on B200: C2 4%
// and C5 2.3x slower than the default -- the distance read filters most
// atomics, and the atomics cost more than the reads.  Off.
#ifndef MB_SSSP_SNAPSHOT
#define MB_SSSP_SNAPSHOT 0
#endif
// The bitmap-output push's neighbour-distance check through L1 (a cached
// copy can only be higher than the current distance -- distances only drop
// -- so a stale hit costs a spurious atomicMin and frontier bit, never a
// missed relaxation).  Measurement switch.
#ifndef MB_SSSP_DIST_L1
#define MB_SSSP_DIST_L1 0
#endif
// 128-bit col/wt loads in the edge-balanced push (needs 4 edges per thread:
// MB_TILE_EDGES=1024).  Measured against the scalar loads; off.
#ifndef MB_PUSH_VEC4
#define MB_PUSH_VEC4 0
#endif

// kBmOut: instead of claiming each improved vertex (an atomic with a
// result) and appending it to the next queue, set its bit in a.nbm with a
// fire-and-forget atomicOr; k_nbm2q then builds the next queue.
template <bool kBmOut, bool kBulk = false>
__device__ __forceinline__ void work_push_edge_q(const SsspArgs &a, PushSmem &sm) {
    uint32_t parity = 0;
    int32_t *s_row = sm.row;
    float *s_du = sm.du;
    BlockQueue &bq = sm.bq;
    if (threadIdx.x == 0) {
        bq.n = 0;
        if (kBulk) {
            mbar_init(&sm.bar, 1);
            fence_barrier_init();
        }
    }
    __syncthreads();
    Ctrl *c = a.f.ctrl;
    const int cur = c->cur, nxt = cur ^ 1;
    const uint64_t q = c->q[cur];
    const uint32_t n = (uint32_t)(q >> 32), m = (uint32_t)q;
    const int32_t sv = c->step + 1;
    // near-far: relaxations to >= thresh go to the far pile
    const float thresh = c->p.delta > 0.f ? c->thresh : 3.0e38f;
    const int32_t *qv = pick(a.f.qv, cur);
    const uint32_t *qo = pick(a.f.qo, cur);
    const int32_t *tf = pick(a.f.tf, cur);
    const uint32_t tiles = (m + kTile - 1) / kTile;
    const uint32_t bulk_polls = c->p.wait_polls >= 0 ? (uint32_t)min(c->p.wait_polls, (int64_t)kBulkSpins) : kBulkSpins;
    uint32_t cn = 0;
    bool stop = false;  // block-uniform: a bulk copy timed out
    for (uint32_t t = blockIdx.x; t < tiles && !stop; t += gridDim.x) {
        const uint32_t c0 = t * kTile;
        uint32_t c1 = min(c0 + kTile, m);
        const int32_t i0 = tf[t];
        const int32_t i1 = (t + 1 < tiles) ? tf[t + 1] : (int32_t)n - 1;
        int k = i1 - i0 + 1;
        // entries [a0, a1) with a0 = i0 rounded down, a1 = i1 + 1 rounded up
        // to 4 entries (16 bytes); the queues hold V + 8 entries
        const int32_t a0 = i0 & ~3, a1 = (i1 + 1 + 3) & ~3;
        if (kBulk && threadIdx.x == 0) {
            const uint32_t bytes = 4u * (uint32_t)(a1 - a0);  // <= 4 * kStage
            fence_proxy_async_smem();  // the last tile's reads of the stage buffers came first
            mbar_arrive_expect_tx(&sm.bar, 2 * bytes);
            bulk_g2s(sm.qo_st, qo + a0, bytes, &sm.bar);
            bulk_g2s(sm.qv_st, qv + a0, bytes, &sm.bar);
        }
        // the same for every thread
        const bool staged = !kBulk || mbar_wait(&sm.bar, parity, bulk_polls);
        if (!staged) {  // record it, let the copies finish (a wait with the
            // full budget: no copy may still be landing when the CTA moves
            // on), and relax nothing more
            if (threadIdx.x == 0) atomicOr(&c->err, ERR_BULK);
            mbar_wait(&sm.bar, parity);
            k = 0;
            c1 = c0;
            stop = true;
        }
        parity ^= 1u;
        const uint32_t *s_off = sm.qo_st + (kBulk ? i0 - a0 : 0);
        if (kBulk) {
            const int32_t *s_qv = sm.qv_st + (i0 - a0);
            for (int j = threadIdx.x; j < k; j += blockDim.x) {
                const int32_t u = s_qv[j];
                s_row[j] = a.row[u];
                s_du[j] = ld_dist(a, u);
            }
        } else {
            for (int j = threadIdx.x; j < k; j += blockDim.x) {
                const int32_t u = qv[i0 + j];
                sm.qo_st[j] = qo[i0 + j];
                s_row[j] = a.row[u];
                s_du[j] = ld_dist(a, u);
            }
        }
        __syncthreads();
        // the thread's kTileItems CONSECUTIVE edges: one binary search for the
        // first, then walk; all loads first, then the relaxations
        int32_t v[kTileItems];
        float nd[kTileItems], dv[kTileItems];
        bool ok[kTileItems];
        {
            const uint32_t e0 = c0 + threadIdx.x * kTileItems;
            int j = e0 < c1 ? upper_bound_minus1(s_off, k, e0) : 0;
#if MB_PUSH_VEC4
            // 128-bit loads of col and wt where the thread's 4 edges lie in one
            // vertex's list and start on a 16-byte boundary; scalar elsewhere
            static_assert(kTileItems == 4, "MB_PUSH_VEC4 needs 4 edges per thread");
            bool vec_done = false;
            if (e0 + 3 < c1 && (j + 1 >= k || s_off[j + 1] > e0 + 3)) {
                const int32_t e = s_row[j] + (int32_t)(e0 - s_off[j]);
                if ((e & 3) == 0) {
                    const int4 c4 = __ldg(reinterpret_cast<const int4 *>(a.col + e));
                    const float4 w4 = __ldg(reinterpret_cast<const float4 *>(a.wt + e));
                    const float du = s_du[j];
                    v[0] = c4.x; v[1] = c4.y; v[2] = c4.z; v[3] = c4.w;
                    nd[0] = du + w4.x; nd[1] = du + w4.y; nd[2] = du + w4.z; nd[3] = du + w4.w;
#pragma unroll
                    for (int r = 0; r < 4; r++) ok[r] = true;
                    vec_done = true;
                }
            }
            if (!vec_done)
#endif
#pragma unroll
            for (int r = 0; r < kTileItems; r++) {
                const uint32_t e_idx = e0 + r;
                ok[r] = e_idx < c1;
                v[r] = 0;
                nd[r] = 0.f;
                if (ok[r]) {
                    while (j + 1 < k && s_off[j + 1] <= e_idx) j++;
                    const int32_t e = s_row[j] + (int32_t)(e_idx - s_off[j]);
                    v[r] = __ldg(&a.col[e]);
                    nd[r] = s_du[j] + __ldg(&a.wt[e]);
                }
            }
        }
#if MB_SSSP_MATCH
        // same-destination relaxations of a warp combined: one distance read
        // and one reduction per distinct destination (R-MAT sends many edges
        // to the same hubs); the lowest lane of each group keeps the minimum
        if (kBmOut) {
            const int lane = threadIdx.x & 31;
#pragma unroll
            for (int r = 0; r < kTileItems; r++) {
                const unsigned act = __ballot_sync(0xffffffffu, ok[r]);
                if (ok[r]) {
                    const unsigned peers = __match_any_sync(act, v[r]);
                    nd[r] = __uint_as_float(__reduce_min_sync(peers, __float_as_uint(nd[r])));
                    ok[r] = lane == __ffs(peers) - 1;
                }
            }
        }
#endif
#if MB_SSSP_SNAPSHOT
        if (kBmOut && thresh > 1e38f) {  // block-uniform
#pragma unroll
            for (int r = 0; r < kTileItems; r++)
                if (ok[r]) atomicMin((unsigned *)&a.dist[v[r]], __float_as_uint(nd[r]));
            __syncthreads();  // the tile's shared entries are reloaded next
            continue;
        }
#endif
#pragma unroll
        for (int r = 0; r < kTileItems; r++)
            dv[r] = ok[r] ? ((MB_SSSP_DIST_L1 && kBmOut) ? __ldca(&a.dist[v[r]]) : ld_dist(a, v[r])) : 0.f;
        if (kBmOut) {
#pragma unroll
            for (int r = 0; r < kTileItems; r++) {
                bool to_far = false;
                if (ok[r] && nd[r] < dv[r]) {
                    atomicMin((unsigned *)&a.dist[v[r]], __float_as_uint(nd[r]));
                    if (nd[r] >= thresh) to_far = true;
                    else atomicOr(&a.nbm[v[r] >> 5], 1u << (v[r] & 31));
                }
                far_push(a, c, to_far, v[r]);
            }
            __syncthreads();  // the tile's shared entries are reloaded next
            continue;
        }
#pragma unroll
        for (int r = 0; r < kTileItems; r++) {
            bool own = false, to_far = false;
            uint32_t deg = 0;
            if (ok[r] && nd[r] < dv[r]) {
                // fire-and-forget minimum; v is queued whenever this candidate
                // beat the distance just read -- if another thread lowered it
                // further meanwhile, v is queued anyway, which is harmless
                atomicMin((unsigned *)&a.dist[v[r]], __float_as_uint(nd[r]));
                if (nd[r] >= thresh) {
                    to_far = true;
                } else if (mark(a, v[r], sv)) {
                    deg = (uint32_t)a.f.outdeg[v[r]];
                    own = true;
                    cn++;
                }
            }
            bq_push(bq, own && deg > 0, v[r], deg);
            far_push(a, c, to_far, v[r]);
        }
        bq_flush(bq, &c->q[nxt], pick(a.f.qv, nxt), pick(a.f.qo, nxt), pick(a.f.tf, nxt));
    }
    flush_counts(c, cn, 0);  // ends with a CTA barrier
    if (kBulk && threadIdx.x == 0) mbar_inval(&sm.bar);  // a later call initialises it again
}

template <bool kBulk>
__global__ void __launch_bounds__(kPushThreads) k_push_edge_q(SsspArgs a) {
    __shared__ PushSmem sm;
    count_launch(a.f.ctrl);
    work_push_edge_q<false, kBulk>(a, sm);
}

template <bool kBulk>
__global__ void __launch_bounds__(kPushThreads) k_push_edge_bm(SsspArgs a) {
    __shared__ PushSmem sm;
    count_launch(a.f.ctrl);
    work_push_edge_q<true, kBulk>(a, sm);
}

// After k_push_edge_bm: next-frontier bitmap -> next queue (with the
// claimed-vertex count), clearing the bitmap.  Each round a block takes one
// word per warp and publishes the round's vertices with ONE atomic (the
// block queue) instead of one per warp on the same counter.  Every vertex
// taken is stamped as updated in this superstep, as the claim of the queue
// path does (schedule 6 sends from the stamped vertices).
__global__ void __launch_bounds__(kPushThreads) k_nbm2q(SsspArgs a) {
    __shared__ BlockQueue bq;
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const int nxt = c->cur ^ 1;
    const int32_t sv = c->step + 1;
    const int lane = threadIdx.x & 31;
    const int64_t wpb = blockDim.x >> 5;
    if (threadIdx.x == 0) bq.n = 0;
    __syncthreads();
    uint32_t cn = 0;
    for (int64_t w0 = (int64_t)blockIdx.x * wpb; w0 < a.f.W; w0 += (int64_t)gridDim.x * wpb) {
        const int64_t w = w0 + (threadIdx.x >> 5);
        const int32_t v = (int32_t)(w * 32 + lane);
        const uint32_t word = w < a.f.W ? a.nbm[w] : 0u;
        if (word && lane == 0) a.nbm[w] = 0u;
        const bool in = (word >> lane) & 1u;
        uint32_t deg = 0;
        if (in) {
            deg = (uint32_t)a.f.outdeg[v];
            a.stamp[v] = sv;
            cn++;
        }
        bq_push(bq, in && deg > 0, v, deg);
        bq_flush(bq, &c->q[nxt], pick(a.f.qv, nxt), pick(a.f.qo, nxt), pick(a.f.tf, nxt));
    }
    flush_counts(c, cn, 0);
}

#if MB_SSSP_SNAPSHOT
__global__ void k_snap(SsspArgs a) {
    count_launch(a.f.ctrl);
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < a.f.V;
         v += (int64_t)gridDim.x * blockDim.x)
        a.dprev[v] = __ldcg(&a.dist[v]);
}

// After the snapshot push: the vertices whose distance dropped -> next queue.
__global__ void __launch_bounds__(kPushThreads) k_snap2q(SsspArgs a) {
    __shared__ BlockQueue bq;
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const int nxt = c->cur ^ 1;
    const int32_t sv = c->step + 1;
    if (threadIdx.x == 0) bq.n = 0;
    __syncthreads();
    uint32_t cn = 0;
    const int64_t per = (int64_t)blockDim.x;
    for (int64_t v0 = (int64_t)blockIdx.x * per; v0 < a.f.V; v0 += (int64_t)gridDim.x * per) {
        const int64_t v = v0 + threadIdx.x;
        bool in = false;
        uint32_t deg = 0;
        if (v < a.f.V && __ldcg(&a.dist[v]) < a.dprev[v]) {
            in = true;
            deg = (uint32_t)a.f.outdeg[v];
            a.stamp[v] = sv;
            cn++;
        }
        bq_push(bq, in && deg > 0, (int32_t)v, deg);
        bq_flush(bq, &c->q[nxt], pick(a.f.qv, nxt), pick(a.f.qo, nxt), pick(a.f.tf, nxt));
    }
    flush_counts(c, cn, 0);
}
#endif

// schedule 1: push, warp-per-vertex for lists >= 32, warp-wide gather below
__global__ void __launch_bounds__(kPushThreads) k_push_warp_q(SsspArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const int cur = c->cur, nxt = cur ^ 1;
    const uint32_t n = (uint32_t)(c->q[cur] >> 32);
    const int32_t sv = c->step + 1;
    const int32_t *qv = pick(a.f.qv, cur);
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    auto visit = [&](bool valid, int32_t e, float du) {
        bool own = false;
        int32_t v = 0;
        uint32_t deg = 0;
        if (valid) {
            v = a.col[e];
            if (relax(a, v, du + a.wt[e], sv)) {
                deg = (uint32_t)a.f.outdeg[v];
                own = true;
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
        float du = 0.f;
        if (i < n) {
            u = qv[i];
            st = a.row[u];
            deg = (uint32_t)a.f.outdeg[u];
            du = ld_dist(a, u);
        }
        unsigned big = __ballot_sync(0xffffffffu, deg >= 32);
        while (big) {
            const int l = __ffs(big) - 1;
            big &= big - 1;
            const int32_t bst = __shfl_sync(0xffffffffu, st, l);
            const uint32_t bdeg = __shfl_sync(0xffffffffu, deg, l);
            const float bdu = __shfl_sync(0xffffffffu, du, l);
            for (uint32_t k = 0; k < bdeg; k += 32)
                visit(k + lane < bdeg, bst + (int32_t)(k + lane), bdu);
        }
        const uint32_t sd = deg < 32 ? deg : 0u;
        const uint32_t incl = warp_incl_scan_u32(sd);
        warp_gather(incl, sd, st, [&](bool valid, int32_t e, int owner) {
            const float odu = __shfl_sync(0xffffffffu, du, owner);
            visit(valid, e, odu);
        });
    }
    flush_counts(c, cn, 0);
}

// an improved vertex joins the bitmap frontier of the next superstep
__device__ __forceinline__ void improve_bm(const SsspArgs &a, uint32_t *next, int32_t v, float nd,
                                           int32_t sv, uint32_t &cn, uint64_t &cm) {
    if (relax(a, v, nd, sv)) {
        atomicOr(&next[v >> 5], 1u << (v & 31));
        cn++;
        cm += (uint32_t)a.f.outdeg[v];
    }
}

// schedules 2 and 3: push over a bitmap frontier; one warp per word
template <bool kEdgeBalanced>
__global__ void __launch_bounds__(kPushThreads) k_push_bm(SsspArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const uint32_t *front = pick(a.f.bm, c->bcur);
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t sv = c->step + 1;
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
        const float du = in ? ld_dist(a, u) : 0.f;
        if (kEdgeBalanced) {
            const uint32_t incl = warp_incl_scan_u32(deg);
            warp_gather(incl, deg, st, [&](bool valid, int32_t e, int owner) {
                const float odu = __shfl_sync(0xffffffffu, du, owner);
                if (valid) improve_bm(a, next, a.col[e], odu + a.wt[e], sv, cn, cm);
            });
        } else {
            unsigned live = __ballot_sync(0xffffffffu, deg > 0);
            while (live) {
                const int l = __ffs(live) - 1;
                live &= live - 1;
                const int32_t bst = __shfl_sync(0xffffffffu, st, l);
                const uint32_t bdeg = __shfl_sync(0xffffffffu, deg, l);
                const float bdu = __shfl_sync(0xffffffffu, du, l);
                for (uint32_t k = lane; k < bdeg; k += 32) {
                    const int32_t e = bst + (int32_t)k;
                    improve_bm(a, next, a.col[e], bdu + a.wt[e], sv, cn, cm);
                }
            }
        }
    }
    flush_counts(c, cn, cm);
}

// Pull epilogue of one word: lanes whose `found` is set lowered their vertex
// to `best`; the warp writes the next-frontier word (it owns it).
__device__ __forceinline__ void pull_commit(const SsspArgs &a, uint32_t *next, int64_t w, int32_t v,
                                            bool found, float best, int32_t sv, uint32_t &cn,
                                            uint64_t &cm) {
    const uint32_t mask = __ballot_sync(0xffffffffu, found);
    if ((threadIdx.x & 31) == 0) next[w] = mask;
    if (found) {
        a.dist[v] = best;
        a.stamp[v] = sv;
        cn++;
        cm += (uint32_t)a.f.outdeg[v];
    }
}

// schedules 4 and 7: pull, edge-streamed.  A warp owns 32 consecutive
// vertices, whose in-edges are contiguous in the reverse CSR; it streams them
// 32 at a time (coalesced rcol/rwt loads), keeps the candidates dist[u]+w of
// frontier sources (schedule 7: every source), and min-combines each into its
// destination's slot with a shared-memory atomicMin on the float bits
// (non-negative floats order like uint32).  The owner of an edge is found by
// binary search over the group's 33 offsets.  Hubs stream at full warp width.
template <bool kAllEdges>
__device__ __forceinline__ void work_pull_stream(const SsspArgs &a) {
    constexpr int kWarps = 256 / 32;
    __shared__ uint32_t s_best[kWarps][32];
    __shared__ int32_t s_off[kWarps][33];
    Ctrl *c = a.f.ctrl;
    const uint32_t *front = pick(a.f.bm, c->bcur);
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t sv = c->step + 1;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t *best = s_best[wid];
    int32_t *off = s_off[wid];
    const int64_t warps = (int64_t)gridDim.x * kWarps;
    uint32_t cn = 0;
    uint64_t cm = 0;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.f.W; w += warps) {
        const int32_t vb = (int32_t)(w * 32);
        const int32_t v = vb + lane;
        const bool valid = v < a.f.V;
        off[lane] = a.rrow[min(v, a.f.V)];
        if (lane == 0) off[32] = a.rrow[min(vb + 32, a.f.V)];
        const float cur_d = valid ? ld_dist(a, v) : 0.f;
        best[lane] = __float_as_uint(valid ? cur_d : 3.0e38f);
        __syncwarp();
        const int32_t g0 = off[0], g1 = off[32];
        for (int32_t j = g0 + lane; j < g1; j += 32) {
            const int32_t u = a.rcol[j];
            if (kAllEdges || test_bit(front, u)) {
                const float cand = ld_dist(a, u) + a.rwt[j];
                int lo = 0, hi = 32;  // last slot whose offset <= j
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (off[mid] <= j) lo = mid; else hi = mid;
                }
                atomicMin(&best[lo], __float_as_uint(cand));
            }
        }
        __syncwarp();
        const float b = __uint_as_float(best[lane]);
        pull_commit(a, next, w, v, valid && b < cur_d, b, sv, cn, cm);
        __syncwarp();
    }
    flush_counts(c, cn, cm);
}

template <bool kAllEdges>
__global__ void __launch_bounds__(256) k_pull_stream(SsspArgs a) {
    count_launch(a.f.ctrl);
    work_pull_stream<kAllEdges>(a);
}

// schedule 5: pull, warp-per-vertex.  mode 1: full Bellman-Ford over every
// in-edge (schedule 7), no frontier test.
template <bool kAllEdges>
__global__ void __launch_bounds__(256) k_pull_warp(SsspArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const uint32_t *front = pick(a.f.bm, c->bcur);
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t sv = c->step + 1;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    uint64_t cm = 0;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.f.W; w += warps) {
        const uint32_t valid = tail_mask(w, a.f.V);
        float mybest = 0.f, mycur = 0.f;
        for (int l = 0; l < 32; l++) {
            if (!((valid >> l) & 1u)) break;
            const int32_t v = (int32_t)(w * 32 + l);
            const int32_t jb = a.rrow[v], je = a.rrow[v + 1];
            float m = 3.0e38f;
            for (int32_t b = jb + lane; b < je; b += 32) {
                const int32_t u = a.rcol[b];
                if (kAllEdges || test_bit(front, u)) m = fminf(m, ld_dist(a, u) + a.rwt[b]);
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == l) {
                mycur = ld_dist(a, v);
                mybest = fminf(mycur, m);
            }
        }
        const int32_t v = (int32_t)(w * 32 + lane);
        pull_commit(a, next, w, v, ((valid >> lane) & 1u) && mybest < mycur, mybest, sv, cn, cm);
    }
    flush_counts(c, cn, cm);
}

// schedule 6, step 1 (InitMessageBuffer, SSSP/InitMessage.h:4-9): msg[] = FLT_MAX
__global__ void k_msg_fill(SsspArgs a) {
    count_launch(a.f.ctrl);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.f.E;
         i += (int64_t)gridDim.x * blockDim.x)
        a.msg[i] = 3.402823466e+38f;
}

// schedule 6, step 2 (ssspEdgeProcAA, SSSP/UserOperators.h:10-29): every
// vertex updated in the last superstep writes dist+w into its edges' slots
__global__ void k_msg_send(SsspArgs a) {
    count_launch(a.f.ctrl);
    const int32_t s = a.f.ctrl->step;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < a.f.V;
         v += (int64_t)gridDim.x * blockDim.x) {
        if (a.stamp[v] != s) continue;
        const float d = a.dist[v];
        for (int32_t e = a.row[v]; e < a.row[v + 1]; e++) a.msg[a.mslot[e]] = d + a.wt[e];
    }
}

// schedule 6, step 3 (segmented min + UpdateVertex, SSSP/UserOperators.h:151-168):
// the combined message of v is the min of its slots [rrow[v], rrow[v+1]).
__global__ void __launch_bounds__(256) k_msg_combine_update(SsspArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    uint32_t *next = pick(a.f.bm, c->bcur ^ 1);
    const int32_t sv = c->step + 1;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    uint64_t cm = 0;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < a.f.W; w += warps) {
        const int32_t v = (int32_t)(w * 32 + (threadIdx.x & 31));
        bool found = false;
        float m = 3.402823466e+38f, cur_d = 0.f;
        if (v < a.f.V) {
            for (int32_t i = a.rrow[v]; i < a.rrow[v + 1]; i++) m = fminf(m, a.msg[i]);
            cur_d = a.dist[v];
            found = m < cur_d;
        }
        pull_commit(a, next, w, v, found, m, sv, cn, cm);
    }
    flush_counts(c, cn, cm);
}

// Tail over a frontier kept in global memory (the queue path): used when
// near-far buckets are on (their far pile lives in global memory).
__device__ void tail_global(const SsspArgs &a, int cap, uint32_t *s_off, int32_t *s_row, float *s_du,
                            int &s_go) {
    Ctrl *c = a.f.ctrl;  // the shared-memory shadow (plain loads)
    for (;;) {
        const int cur = c->cur, nxt = cur ^ 1;
        const unsigned long long q = c->q[cur];
        const uint32_t n = (uint32_t)(q >> 32), m = (uint32_t)q;
        const int32_t sv = c->step + 1;
        const float delta = c->p.delta;
        const float thresh = delta > 0.f ? c->thresh : 3.0e38f;
        const int32_t *qv = pick(a.f.qv, cur);
        const uint32_t *qo = pick(a.f.qo, cur);
        for (uint32_t j = threadIdx.x; j < n; j += kTailThreads) {
            const int32_t u = qv[j];
            s_off[j] = qo[j];
            s_row[j] = a.row[u];
            s_du[j] = ld_dist(a, u);
        }
        __syncthreads();
        uint32_t cn = 0;
        for (uint32_t base = 0; base < m; base += kTailThreads) {
            const uint32_t e_idx = base + threadIdx.x;
            bool own = false, to_far = false;
            int32_t v = 0;
            uint32_t deg = 0;
            if (e_idx < m) {
                const int j = upper_bound_minus1(s_off, (int)n, e_idx);
                const int32_t e = s_row[j] + (int32_t)(e_idx - s_off[j]);
                v = __ldg(&a.col[e]);
                const float nd = s_du[j] + __ldg(&a.wt[e]);
                if (lower(a, v, nd)) {
                    if (nd >= thresh) {
                        to_far = true;
                    } else if (mark(a, v, sv)) {
                        deg = (uint32_t)a.f.outdeg[v];
                        own = true;
                        cn++;
                    }
                }
            }
            enqueue_warp(own && deg > 0, v, deg, &c->q[nxt], pick(a.f.qv, nxt), pick(a.f.qo, nxt),
                         pick(a.f.tf, nxt));
            far_push(a, c, to_far, v);
        }
        flush_counts(c, cn, 0);
        __syncthreads();
        if (threadIdx.x == 0) {
            finish_superstep<false>(c, APP_SSSP, a.f.V, a.f.E, FMT_QUEUE);
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
}

// Exclusive scan of x[0..n) in shared memory by the whole CTA (n <= 8 *
// blockDim.x); returns the total.  Uses the 32-entry s_warp scratch.
__device__ uint32_t block_excl_scan(uint32_t *x, uint32_t n, uint32_t *s_warp) {
    constexpr int kPer = kSTailCap / kTailThreads;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t i0 = threadIdx.x * kPer;
    uint32_t loc[kPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        loc[k] = i0 + k < n ? x[i0 + k] : 0u;
        sum += loc[k];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t t = lane < nw ? s_warp[lane] : 0u, ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += y;
        }
        if (lane < nw) s_warp[lane] = ti - t;  // exclusive
        if (lane == 31) s_warp[32] = ti;      // total
    }
    __syncthreads();
    uint32_t off = s_warp[wid] + incl - sum;
#pragma unroll
    for (int k = 0; k < kPer; k++)
        if (i0 + k < n) {
            x[i0 + k] = off;
            off += loc[k];
        }
    const uint32_t total = s_warp[32];
    __syncthreads();
    return total;
}

// Persistent small-frontier tail with the frontier in SHARED memory: ONE CTA
// runs consecutive supersteps of schedule 0 while the frontier stays within
// kTailEntries vertices and p.tail_edges (<= kSTailCap) out-edges.  Per
// superstep only three dependent global round trips remain: the frontier's
// distances, its edges (column, weight), the destinations' distances.  An
// improving relaxation issues a fire-and-forget atomicMin and inserts the
// destination into a shared-memory hash set (the dedup that the global claim
// does elsewhere; the CTA is the only one running).  The control block is
// kept current every superstep (same bookkeeping, same decisions as the
// other paths); the global queue is written only when the tail ends, with
// the stamps that mark its vertices as updated.
__device__ void tail_smem(const SsspArgs &a, int cap, char *smem, int &s_go) {
    Ctrl *c = a.f.ctrl;
    int32_t *s_hash = (int32_t *)smem;                       // kSTailCap * 2
    int32_t *s_q = s_hash + 2 * kSTailCap;                   // kSTailCap
    int32_t *s_row = s_q + kSTailCap;                        // kSTailCap
    uint32_t *s_deg = (uint32_t *)(s_row + kSTailCap);       // kSTailCap (degree, then offset)
    float *s_du = (float *)(s_deg + kSTailCap);              // kTailEntries
    uint32_t *s_warp = (uint32_t *)(s_du + kTailEntries);    // 33
    __shared__ uint32_t s_n, s_m;
    constexpr int32_t kEmpty = -1;
    constexpr uint32_t kHashMask = 2 * kSTailCap - 1;
    for (uint32_t i = threadIdx.x; i < 2 * kSTailCap; i += kTailThreads) s_hash[i] = kEmpty;
    // the frontier from the global queue
    {
        const int cur = c->cur;
        const unsigned long long q = c->q[cur];
        const uint32_t n = (uint32_t)(q >> 32);
        const int32_t *qv = pick(a.f.qv, cur);
        for (uint32_t j = threadIdx.x; j < n; j += kTailThreads) {
            const int32_t u = qv[j];
            s_q[j] = u;
            const int32_t r0 = a.row[u];
            s_row[j] = r0;
            s_deg[j] = (uint32_t)(a.row[u + 1] - r0);
        }
        if (threadIdx.x == 0) s_n = n;
        __syncthreads();
    }
    for (;;) {
        const uint32_t n = s_n;
        for (uint32_t j = threadIdx.x; j < n; j += kTailThreads) s_du[j] = ld_dist(a, s_q[j]);
        const uint32_t m = block_excl_scan(s_deg, n, s_warp);  // s_deg -> offsets
        // relax every frontier edge: each thread takes kTR consecutive edges
        // (one search, then a walk) and issues all their loads before using
        // any, so one round trip covers the whole frontier (m <= kSTailCap)
        constexpr int kTR = kSTailCap / kTailThreads;
        bool reduced = false;
        {
            const uint32_t e0 = threadIdx.x * kTR;
            int32_t v[kTR];
            float nd[kTR], dv[kTR];
            int j = e0 < m ? upper_bound_minus1(s_deg, (int)n, e0) : 0;
#pragma unroll
            for (int r = 0; r < kTR; r++) {
                const uint32_t e_idx = e0 + r;
                v[r] = -1;
                nd[r] = 0.f;
                if (e_idx < m) {
                    while (j + 1 < (int)n && s_deg[j + 1] <= e_idx) j++;
                    const int32_t e = s_row[j] + (int32_t)(e_idx - s_deg[j]);
                    v[r] = __ldg(&a.col[e]);
                    nd[r] = s_du[j] + __ldg(&a.wt[e]);
                }
            }
#pragma unroll
            for (int r = 0; r < kTR; r++) dv[r] = v[r] >= 0 ? ld_dist(a, v[r]) : 0.f;
#pragma unroll
            for (int r = 0; r < kTR; r++) {
                if (v[r] >= 0 && nd[r] < dv[r]) {
                    atomicMin((unsigned *)&a.dist[v[r]], __float_as_uint(nd[r]));  // no result needed
                    reduced = true;
                    uint32_t h = ((uint32_t)v[r] * 2654435761u) & kHashMask;
                    for (;;) {  // the set holds <= m <= kSTailCap < 2 * kSTailCap slots
                        const int32_t old = atomicCAS(&s_hash[h], kEmpty, v[r]);
                        if (old == kEmpty || old == v[r]) break;
                        h = (h + 1) & kHashMask;
                    }
                }
            }
        }
        // the next superstep reads these distances (at L2) from other threads:
        // the fire-and-forget reductions must be performed first, which the
        // CTA barrier alone does not order
        if (reduced) __threadfence();
        if (threadIdx.x == 0) {
            s_n = 0;
            s_m = 0;
        }
        __syncthreads();
        // the set -> the next frontier (clearing the set).  As the queue path
        // does, only vertices with out-edges join it: the merge-path kernels
        // size their per-tile staging on at least one edge per entry.
        uint32_t mloc = 0;
        for (uint32_t i = threadIdx.x; i < 2 * kSTailCap; i += kTailThreads) {
            const int32_t v = s_hash[i];
            if (v != kEmpty) {
                s_hash[i] = kEmpty;
                const int32_t r0 = a.row[v];
                const uint32_t d = (uint32_t)(a.row[v + 1] - r0);
                if (d > 0) {
                    const uint32_t pos = atomicAdd(&s_n, 1u);
                    s_q[pos] = v;
                    s_row[pos] = r0;
                    s_deg[pos] = d;
                    mloc += d;
                }
            }
        }
        mloc = warp_sum(mloc);
        if ((threadIdx.x & 31) == 0 && mloc) atomicAdd(&s_m, mloc);
        __syncthreads();
        const uint32_t n2 = s_n, m2 = s_m;
        if (threadIdx.x == 0) {
            const int nxt = c->cur ^ 1;
            c->q[nxt] = ((unsigned long long)n2 << 32) | m2;
            c->acc_n = n2;
            c->acc_m = 0;
            finish_superstep<false>(c, APP_SSSP, a.f.V, a.f.E, FMT_QUEUE);
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
    // publish the frontier to the global queue (offsets, tile starts, stamps)
    const uint32_t n = s_n;
    if (n == 0) return;
    const int cur = c->cur;  // finish_superstep made the next queue current
    const int32_t sv = c->step;
    block_excl_scan(s_deg, n, s_warp);
    int32_t *qv = pick(a.f.qv, cur);
    uint32_t *qo = pick(a.f.qo, cur);
    int32_t *tf = pick(a.f.tf, cur);
    const uint32_t m = (uint32_t)c->q[cur];
    for (uint32_t i = threadIdx.x; i < n; i += kTailThreads) {
        const int32_t v = s_q[i];
        const uint32_t off = s_deg[i];
        const uint32_t d = (i + 1 < n ? s_deg[i + 1] : m) - off;  // >= 1
        qv[i] = v;
        qo[i] = off;
        a.stamp[v] = sv;
        for (uint32_t t = (off + kTile - 1) / kTile; t <= (off + d - 1) / kTile; t++) tf[t] = (int32_t)i;
    }
}

#ifndef MB_TAIL_MIN_BLOCKS
#define MB_TAIL_MIN_BLOCKS 1
#endif
__global__ void __launch_bounds__(kTailThreads, MB_TAIL_MIN_BLOCKS) k_tail(SsspArgs a, int cap) {
    count_launch(a.f.ctrl);
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_go;
    __shared__ Ctrl s_ctrl;  // shadow of the control block (plain loads only)
    Ctrl *const gc = a.f.ctrl;
    ctrl_shadow_in(&s_ctrl, gc);
    SsspArgs sa = a;
    sa.f.ctrl = &s_ctrl;
    if (s_ctrl.p.delta > 0.f) {
        tail_global(sa, cap, (uint32_t *)smem, (int32_t *)(smem + 4 * kTailEntries),
                    (float *)(smem + 8 * kTailEntries), s_go);
    } else {
        tail_smem(sa, cap, smem, s_go);
    }
    // every superstep this kernel ran is finished already
    if (threadIdx.x == 0) s_ctrl.pending = 0;
    ctrl_shadow_out(gc, &s_ctrl);
}

// Near-far split: the threshold was just raised (by delta, and past the
// least distance the last split kept); every far-pile vertex now below it
// joins the near queue, the rest move to the other pile, and the least
// distance kept is recorded for the next raise.
__device__ __forceinline__ void work_far_split(const SsspArgs &a) {
    Ctrl *c = a.f.ctrl;
    const int f = c->fcur;
    const uint32_t n = c->far_n[f];
    const int32_t *src = pick(a.far, f);
    const float thresh = c->thresh, thresh_prev = c->thresh_prev;
    float kept_min = __uint_as_float(0x7f800000u);  // least distance this warp keeps parked
    const int nxt = c->cur ^ 1;
    const int32_t sv = c->step + 1;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    uint32_t cn = 0;
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < n;
         base += warps * 32) {
        const int64_t i = base + lane;
        bool near = false, keep = false;
        int32_t v = 0;
        uint32_t deg = 0;
        if (i < n) {
            v = src[i];
            const float d = ld_dist(a, v);
            if (d < thresh) {
                // leaves the piles; a kept vertex keeps its bit, the pile it
                // moves to becomes the one being filled.  Below the previous
                // threshold it was expanded at this distance already (it got
                // there through the near queue), so it is dropped.
                atomicAnd(&a.farbm[v >> 5], ~(1u << (v & 31)));
                if (d >= thresh_prev && mark(a, v, sv)) {
                    deg = (uint32_t)a.f.outdeg[v];
                    near = true;
                    cn++;
                }
            } else {
                keep = true;
                kept_min = fminf(kept_min, d);
            }
        }
        enqueue_warp(near && deg > 0, v, deg, &c->q[nxt], pick(a.f.qv, nxt), pick(a.f.qo, nxt),
                     pick(a.f.tf, nxt));
        // the kept ones go to the other pile
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (mask) {
            const int leader = __ffs(mask) - 1;
            uint32_t b = 0;
            if (lane == leader) b = atomicAdd(&c->far_n[f ^ 1], (uint32_t)__popc(mask));
            b = __shfl_sync(0xffffffffu, b, leader);
            if (keep) pick(a.far, f ^ 1)[b + __popc(mask & lanemask_lt())] = v;
        }
    }
    // the next raise skips to this (distances are non-negative: float bits
    // order like the numbers)
    const unsigned km = __reduce_min_sync(0xffffffffu, __float_as_uint(kept_min));
    if (lane == 0 && km < 0x7f800000u) atomicMin(&c->far_min, km);
    flush_counts(c, cn, 0);
}

__global__ void __launch_bounds__(256) k_far_split(SsspArgs a) {
    count_launch(a.f.ctrl);
    work_far_split(a);
}

// Persistent BSP kernel (cooperative launch, all blocks resident): runs
// consecutive supersteps of schedules 0 and 4 (with their frontier
// conversions) and near-far splits, separated by grid barriers; block 0 does
// each superstep's bookkeeping between two barriers.  Leaves when the next
// superstep needs another schedule, the run is done, or a barrier gives up.
__global__ void __launch_bounds__(kPushThreads) k_persist(SsspArgs a, int cap) {
    __shared__ PushSmem sm;
    Ctrl *c = a.f.ctrl;
    count_launch(c);
    for (;;) {
        const int s = ldg2(&c->sched), mode = ldg2(&c->mode);
        if (s == kSchedSplit) {
            work_far_split(a);
        } else {
            if (!persist_convert(a.f, s, mode)) break;
            if (s == MB_SCHED_PULL_THREAD) work_pull_stream<false>(a);
            else work_push_edge_q<false>(a, sm);
        }
        if (!grid_sync(c)) break;
        persist_bookkeep(a.f, APP_SSSP, cap);
        if (!grid_sync(c)) break;
        if (!ldg2(&c->persist_go)) break;
    }
}

#include "sssp_async.cuh"

__global__ void k_sssp_init(SsspArgs a) {
    count_launch(a.f.ctrl);
    Ctrl *c = a.f.ctrl;
    const int32_t source = c->p.source;
    const int32_t deg = a.f.outdeg[source];
    if (threadIdx.x == 0) {
        a.dist[source] = 0.0f;
        a.stamp[source] = 0;
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
        c->reached = 0;
        c->edges_reached = 0;
        c->work = 0;
        c->pending = 0;
        c->thresh = c->p.delta;
        c->thresh_prev = 0.f;
        c->far_min = 0x7f800000u;
        c->far_n[0] = 0;
        c->far_n[1] = 0;
        c->fcur = 0;
        c->splits = 0;
        c->bar_count = 0;
        c->peaked = 0;
        c->q[1] = 0ull;
        a.as->pt.v = 0ull;
        a.as->mn[0].v = kInfBits;
        a.as->mn[1].v = kInfBits;
        a.as->t0.v = kInfBits;
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
    // the asynchronous kernel's counters (thread 0 set the threshold lines above)
    {
        unsigned long long *w = &a.as->p[0].v;
        constexpr int kWords = (int)(offsetof(AsyncState, pt) / 8);
        for (int i = threadIdx.x; i < kWords; i += blockDim.x) w[i] = 0ull;
        if (threadIdx.x < 2) a.as->idle[threadIdx.x].v = 0ull;
        if (threadIdx.x == 2) a.as->bar.v = 0ull;
        if (threadIdx.x == 3) a.as->abort_.v = 0ull;
    }
    __syncthreads();
    if (threadIdx.x == 0) choose_next(c, APP_SSSP, a.f.V, a.f.E);
}

__global__ void k_fill_dist(SsspArgs a) {
    count_launch(a.f.ctrl);
    float *d = a.dist;
    const int64_t n = a.f.V;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = kMedusaMax;
}

__global__ void k_stats(SsspArgs a) {
    count_launch(a.f.ctrl);
    uint32_t n = 0;
    uint64_t m = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < a.f.V;
         v += (int64_t)gridDim.x * blockDim.x) {
        if (a.dist[v] < kMedusaMax) {
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

// Hop distances of a unit-weight run -> BFS levels (-1 unreached).
__global__ void k_dist_to_level(SsspArgs a, int32_t *level) {
    count_launch(a.f.ctrl);
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < a.f.V;
         v += (int64_t)gridDim.x * blockDim.x) {
        const float d = a.dist[v];
        level[v] = d < kMedusaMax ? (int32_t)d : -1;
    }
}

__global__ void k_weight_sum(const float *w, int64_t E, double *out, unsigned *bad) {
    double t = 0.0;
    unsigned nb = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < E;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float x = w[i];
        t += x;
        nb += !(x >= 0.f);  // negative or NaN
    }
    t = warp_sum(t);
    nb = warp_sum(nb);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, t);
        if (nb) atomicAdd(bad, nb);
    }
}

}  // namespace

uint32_t sssp_bm_push_min(const Context &ctx, const Graph &g) {
    const int64_t t = ctx.tunable[MB_TUNE_SSSP_BM_PUSH_MIN];
    if (t >= 0) return (uint32_t)std::min<int64_t>(t, 0xffffffffll);
    return (uint32_t)std::min<int64_t>(std::max<int64_t>(1 << 20, g.E / 8), 0xffffffffll);
}

void sssp_weight_stats(const Graph &g, double *mean_w, bool *bad) {
    *mean_w = 0.0;
    *bad = false;
    if (g.E == 0) return;
    DevBuf acc;
    acc.reserve(sizeof(double) + sizeof(unsigned));
    MB_CUDA(cudaMemset(acc.p, 0, sizeof(double) + sizeof(unsigned)));
    unsigned *d_bad = (unsigned *)(acc.as<char>() + sizeof(double));
    k_weight_sum<<<grid_for(g.E, 256, 1184), 256>>>(g.wt.as<float>(), g.E, acc.as<double>(), d_bad);
    MB_CHECK_LAUNCH();
    struct {
        double sum;
        unsigned nbad;
    } h;
    MB_CUDA(cudaMemcpy(&h.sum, acc.p, sizeof(double), cudaMemcpyDeviceToHost));
    MB_CUDA(cudaMemcpy(&h.nbad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost));
    acc.release();
    *mean_w = h.sum / (double)g.E;
    *bad = h.nbad != 0;
}

float sssp_default_delta(const Graph &g, double mean_w) {
    if (g.E == 0) return 0.f;
    const double mean_deg = (double)g.E / (double)g.V;
    constexpr double kDeltaWarps = 32.0;
    return (float)(mean_w * kDeltaWarps / std::max(1.0, mean_deg));
}

float sssp_async_delta(const Graph &g, double mean_w) {
    if (g.E == 0) return 0.f;
    const double mean_deg = (double)g.E / (double)g.V;
    return (float)std::max(mean_w, mean_w * 24.0 / std::max(1.0, mean_deg));
}

// Hub chunk tables of the asynchronous kernel for graph g (once).
static void async_chunks(Context &ctx, Graph &g, SsspState &st) {
    if (st.nchunks >= 0) return;
    cudaStream_t s = ctx.stream;
    const int32_t V = g.V;
    if (V == 0) {
        st.nchunks = 0;
        return;
    }
    const int gridV = grid_for(V, 256, ctx.num_sms * 8);
    st.hub_cbase.reserve(sizeof(int32_t) * (size_t)V);
    DevBuf tot;
    tot.reserve(sizeof(uint32_t));
    k_chunk_count<<<gridV, 256, 0, s>>>(g.row.as<int32_t>(), V, st.hub_cbase.as<uint32_t>());
    MB_CHECK_LAUNCH();
    scan_exclusive_u32(ctx, st.hub_cbase.as<uint32_t>(), st.hub_cbase.as<uint32_t>(), V, tot.as<uint32_t>(), s);
    uint32_t nc = 0;
    MB_CUDA(cudaMemcpyAsync(&nc, tot.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    tot.release();
    st.nc32 = (int32_t)((nc + 31) / 32);
    if (nc) {
        const size_t slots = 32 * (size_t)st.nc32;  // chunk positions, holes included
        st.chunk_src.reserve(sizeof(int32_t) * slots);
        st.chunk_rs.reserve(sizeof(int32_t) * slots);
        k_chunk_fill<<<gridV, 256, 0, s>>>(g.row.as<int32_t>(), V, st.hub_cbase.as<int32_t>(), st.nc32,
                                           st.chunk_src.as<int32_t>(), st.chunk_rs.as<int32_t>());
        MB_CHECK_LAUNCH();
        st.adirty.reserve(sizeof(uint32_t) * (((size_t)V + slots + 31) / 32));
        MB_CUDA(cudaStreamSynchronize(s));
    } else {
        st.hub_cbase.release();
    }
    st.nchunks = nc;
}

void run_sssp(Context &ctx, Graph &g, SsspState &st, int32_t source, mb_stats *stats, int phase, int force,
             int *cont, int32_t *bfs_levels, const EmitFn *after) {
    if (bfs_levels && (phase != LOOP_ALL || ctx.persist))
        fail(MB_ERR_INVALID, "asynchronous BFS: whole runs without the persistent grid only");
    st.ensure(g);
    SsspArgs a;
    a.f = st.frontier_args(g, ctx.model(MB_MODEL_SSSP));
    a.row = g.row.as<int32_t>();
    a.col = g.col.as<int32_t>();
    a.rrow = g.rrow.as<int32_t>();
    a.rcol = g.rcol.as<int32_t>();
    a.mslot = g.mslot.as<int32_t>();
    a.wt = g.wt.as<float>();
    a.rwt = g.rwt.as<float>();
    a.dist = st.dist.as<float>();
    a.stamp = st.stamp.as<int32_t>();
    a.msg = st.msg.as<float>();
    a.far[0] = st.far[0].as<int32_t>();
    a.far[1] = st.far[1].as<int32_t>();
    a.farbm = st.farbm.as<uint32_t>();
    a.nbm = st.nbm.as<uint32_t>();
    a.dprev = st.dprev.as<float>();
    a.as = st.as.as<AsyncState>();
    // near-far bucket width: the context's, or a per-graph default
    const float delta = ctx.sssp_delta >= 0.f ? ctx.sssp_delta : st.default_delta;
    // asynchronous relaxation: the tunable, else on unless the near-far
    // buckets or the persistent grid were asked for (fixed and learned
    // policies only -- it is how schedule 0 runs the rest of a traversal; the
    // forced and replay policies name every superstep's schedule;
    // non-negative weights only: with a negative or NaN weight the BSP
    // loop's superstep cap is what ends a run).  A BFS run (bfs_levels) is
    // always asynchronous, with every weight 1 and a threshold step in hops.
    const bool unit = bfs_levels != nullptr;
    const int64_t t_async = ctx.tunable[MB_TUNE_SSSP_ASYNC];
    const bool policy_ok = ctx.schedule_policy == MB_POLICY_FIXED || ctx.schedule_policy == MB_POLICY_LEARNED;
    // On a hub-free graph the default runs the whole traversal in the
    // kernel; on a graph with hubs, the BSP supersteps until the frontier,
    // past its peak, has fewer than max(2^18, E/16) out-edges, and the
    // kernel for that tail, with no threshold (measured on B200: C2 SSSP
    // 1.05 -> 0.98 ms; C5 unchanged, 5.15 ms).
    const bool hub_free = async_by_default(g, false);
    // A near-far width turns the kernel off whatever the tunable says: it
    // starts from the queue frontier only, and vertices parked in the far
    // pile would never be expanded.
    const int32_t async =
        unit ? 1
             : (!policy_ok || !st.weights_ok || delta != 0.f
                    ? 0
                    : (t_async >= 0 ? (int32_t)t_async : (!ctx.persist ? 1 : 0)));
    float async_delta = ctx.tunable[MB_TUNE_ASYNC_DELTA] >= 0 ? (float)ctx.tunable[MB_TUNE_ASYNC_DELTA]
                                                               : (hub_free ? st.async_delta : 0.f);
    if (unit)
        async_delta = ctx.tunable[MB_TUNE_BFS_ASYNC_DELTA] >= 0 ? (float)ctx.tunable[MB_TUNE_BFS_ASYNC_DELTA]
                                                                : kBfsAsyncDelta;
    // made on the first run whether or not it is asynchronous: the pointers
    // below are captured in the run's loop graph, which must not change
    // when a later run switches the kernel on
    async_chunks(ctx, g, st);
    const int64_t nchunks = st.nchunks > 0 ? st.nchunks : 0;
    a.nc32 = nchunks ? st.nc32 : 0;
    a.adirty = nchunks ? st.adirty.as<uint32_t>() : a.nbm;
    a.WA = ((int64_t)g.V + 32 * (int64_t)a.nc32 + 31) / 32;
    a.hub_cbase = st.hub_cbase.as<int32_t>();
    a.chunk_src = st.chunk_src.as<int32_t>();
    a.chunk_rs = st.chunk_rs.as<int32_t>();
    const int64_t t_below = ctx.tunable[MB_TUNE_ASYNC_BELOW];
    const int64_t below_dflt = hub_free ? 0 : std::max<int64_t>(1 << 18, g.E / 16);
    const uint32_t async_below =
        unit ? 0u : (uint32_t)std::min<int64_t>(t_below >= 0 ? t_below : below_dflt, 0xffffffffll);
    if (phase == LOOP_ALL)
        upload_params(ctx, st.ctrl.p, source, unit ? 0.f : delta, sssp_bm_push_min(ctx, g), async, async_delta,
                      async_below);
    if (phase == LOOP_BEGIN) {  // a stepped run: one superstep per call (no persistent kernels)
        const bool tail = ctx.tail, persist = ctx.persist;
        ctx.tail = ctx.persist = false;
        upload_params(ctx, st.ctrl.p, source, delta, sssp_bm_push_min(ctx, g));
        ctx.tail = tail;
        ctx.persist = persist;
    }

    const int grid_push = ctx.num_sms * ctx.blocks_per_sm(MB_TUNE_PUSH_BLOCKS_PER_SM, 8);
    const bool bulk = ctx.tunable[MB_TUNE_BULK_STAGE] > 0;
    const int grid_vtx = ctx.num_sms * ctx.blocks_per_sm(MB_TUNE_VERTEX_BLOCKS_PER_SM, 8);
    const int grid_edge = grid_vtx;
    const int persist_grid = persistent_grid_size(ctx, (const void *)k_persist, kPushThreads);
    const void *async_kernel = unit ? (const void *)k_sssp_async<true> : (const void *)k_sssp_async<false>;
    int async_grid = 0;
    {
        int per_sm = 0;
        MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, async_kernel, kAsyncThreads, 0));
        if (per_sm < 1) fail(MB_ERR_UNSUPPORTED, "asynchronous SSSP kernel does not fit on an SM");
        per_sm = std::min(per_sm, 8);
        if (ctx.tunable[MB_TUNE_ASYNC_BLOCKS_PER_SM] > 0)
            per_sm = std::min(per_sm, (int)ctx.tunable[MB_TUNE_ASYNC_BLOCKS_PER_SM]);
        async_grid = ctx.num_sms * per_sm;
    }
    MB_CUDA(cudaFuncSetAttribute((const void *)k_tail, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kTailSmemBytes));
    LoopSpec sp;
    sp.st = &st;
    sp.fa = a.f;
    // each superstep lowers some distance; with integer distances below 2^24
    // a run cannot need more supersteps than this
    sp.app = APP_SSSP;
    sp.cap = step_cap(ctx, (int64_t)g.V * 4 + 16);
    sp.name = "sssp";
    sp.prologue = [&](cudaStream_t s) {
        k_fill_dist<<<grid_vtx, 256, 0, s>>>(a);
        MB_CUDA(cudaMemsetAsync(a.stamp, 0xff, sizeof(int32_t) * (size_t)a.f.V, s));
        MB_CUDA(cudaMemsetAsync(a.farbm, 0, sizeof(uint32_t) * (size_t)a.f.W, s));
        MB_CUDA(cudaMemsetAsync(a.nbm, 0, sizeof(uint32_t) * (size_t)a.f.W, s));
        if (a.adirty != a.nbm) MB_CUDA(cudaMemsetAsync(a.adirty, 0, sizeof(uint32_t) * (size_t)a.WA, s));
        k_sssp_init<<<1, 256, 0, s>>>(a);
        MB_CHECK_LAUNCH();
    };
    sp.branch = [&](int branch, cudaStream_t s) {
        if (branch == kBranchSplit) {
            k_far_split<<<grid_vtx, 256, 0, s>>>(a);
            MB_CHECK_LAUNCH();
            return;
        }
        if (branch == kBranchTail) {
            k_tail<<<1, kTailThreads, kTailSmemBytes, s>>>(a, sp.cap);
            MB_CHECK_LAUNCH();
            return;
        }
        if (branch == kBranchPersist) {
            launch_cooperative((const void *)k_persist, persist_grid, kPushThreads, s, a, sp.cap);
            return;
        }
        if (branch == kBranchAsync) {
            launch_cooperative(async_kernel, async_grid, kAsyncThreads, s, a, sp.cap);
            return;
        }
        if (branch == kBranchPushSmall) {
            const int grid_small = ctx.num_sms * kSmallPushPerSm;
            if (bulk) k_push_edge_q<true><<<grid_small, kPushThreads, 0, s>>>(a);
            else k_push_edge_q<false><<<grid_small, kPushThreads, 0, s>>>(a);
            MB_CHECK_LAUNCH();
            return;
        }
#if MB_SSSP_SNAPSHOT
        if (branch == kBranchPushBm && delta == 0.f) {
            k_snap<<<grid_vtx, 256, 0, s>>>(a);
            if (bulk) k_push_edge_bm<true><<<grid_push, kPushThreads, 0, s>>>(a);
            else k_push_edge_bm<false><<<grid_push, kPushThreads, 0, s>>>(a);
            k_snap2q<<<grid_vtx, kPushThreads, 0, s>>>(a);
            MB_CHECK_LAUNCH();
            return;
        }
#endif
        if (branch == kBranchPushBm) {
            if (bulk) k_push_edge_bm<true><<<grid_push, kPushThreads, 0, s>>>(a);
            else k_push_edge_bm<false><<<grid_push, kPushThreads, 0, s>>>(a);
            k_nbm2q<<<grid_vtx, kPushThreads, 0, s>>>(a);
            MB_CHECK_LAUNCH();
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
            case MB_SCHED_PUSH_EDGE_QUEUE:
                if (bulk) k_push_edge_q<true><<<grid_push, kPushThreads, 0, s>>>(a);
                else k_push_edge_q<false><<<grid_push, kPushThreads, 0, s>>>(a);
                break;
            case MB_SCHED_PUSH_WARP_QUEUE: k_push_warp_q<<<grid_push, kPushThreads, 0, s>>>(a); break;
            case MB_SCHED_PUSH_EDGE_BITMAP:
                k_bm_clear<<<grid_vtx, 256, 0, s>>>(a.f, 1);
                k_push_bm<true><<<grid_push, kPushThreads, 0, s>>>(a);
                break;
            case MB_SCHED_PUSH_WARP_BITMAP:
                k_bm_clear<<<grid_vtx, 256, 0, s>>>(a.f, 1);
                k_push_bm<false><<<grid_push, kPushThreads, 0, s>>>(a);
                break;
            case MB_SCHED_PULL_THREAD: k_pull_stream<false><<<grid_vtx, 256, 0, s>>>(a); break;
            case MB_SCHED_PULL_WARP: k_pull_warp<false><<<grid_vtx, 256, 0, s>>>(a); break;
            case MB_SCHED_PUSH_UNFUSED:
                k_msg_fill<<<grid_edge, 256, 0, s>>>(a);
                k_msg_send<<<grid_vtx, 256, 0, s>>>(a);
                k_msg_combine_update<<<grid_vtx, 256, 0, s>>>(a);
                break;
            default: k_pull_stream<true><<<grid_vtx, 256, 0, s>>>(a); break;
        }
        MB_CHECK_LAUNCH();
    };
    sp.epilogue = [&](cudaStream_t s) {
        k_stats<<<ctx.num_sms * 4, 256, 0, s>>>(a);
        if (unit) k_dist_to_level<<<grid_vtx, 256, 0, s>>>(a, bfs_levels);
        MB_CHECK_LAUNCH();
    };
    if (after) sp.after = *after;
    run_loop(ctx, sp, stats, phase, force, cont);
}

}  // namespace mb
