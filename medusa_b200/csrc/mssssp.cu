// mssssp.cu -- batched SSSP: up to 32 sources in one traversal.
//
// Distances are stored vertex-major, dist[v*32 + s], so the 32 distances of a
// vertex fill one 128-byte line.  front[v], for a vertex of the current
// queue, is the 32-bit mask of the sources whose distance to v dropped in
// the last superstep (entries of other vertices are stale and never read).
// A warp relaxes one edge
// (u,v,w) for every source at once -- lane s holds source s -- so reading
// and updating dist[v][*] is one coalesced line; the lanes that improved are
// combined with __ballot_sync into v's mask of the next frontier.
// Per source this is the same frontier Bellman-Ford as mb_sssp (integer-
// valued float distances, exact minima), so dist_out[s*V + v] equals 32
// single-source runs bit for bit.  No reference counterpart exists for the
// batching itself.
//
// Near-far buckets (width delta > 0, MB_TUNE_MSS_DELTA): the frontier holds
// only the (vertex, source) pairs whose distance is below a threshold T.
// The push marks each improved pair near or far in the head's 64-bit mask;
// the commit queues the near pairs and moves the far ones into far[v] (the
// vertex joins a far list the first time), and when no near pair is left a
// far pass raises T to the least waiting distance + delta and moves the
// pairs now below it back into the queue.  Each pair is still relaxed until
// no distance drops, so the distances are the same fixpoint; what changes
// is how often an edge is relaxed before its tail's distance is final.
#include <algorithm>
#include <cmath>
#include "mssssp.cuh"
#include "sssp.cuh"

namespace mb {
namespace {

constexpr int kWarpEdges = 32;  // consecutive edges a warp relaxes per pass
constexpr uint32_t kMsInfBits = 0x7f800000u;  // +inf

struct MsCtrl {
    unsigned long long q[2];
    uint32_t touched;
    int32_t cur;
    int32_t supersteps;
    int32_t done;
    unsigned long long work;  // edges relaxed (for all sources of a batch)
    // near-far buckets (delta > 0)
    float T;            // pairs at distance >= T wait in far[v]
    uint32_t fmin;      // float bits: least distance recorded for a parked pair since the last far pass
    int32_t fl;         // the far list that receives newly waiting vertices
    int32_t advance;    // 1: the queue is empty and pairs wait
    uint32_t nfar[2];   // far list lengths
};

struct MsArgs {
    int32_t V;
    int64_t E;
    const int32_t *row, *col, *outdeg;
    const float *wt;
    float *dist;  // [V][32]
    uint32_t *front[2], *nxt;
    unsigned long long *nxt2;  // the same buffer with near-far: far bits << 32 | near bits
    int32_t *touched;
    int32_t *qv[2];
    uint32_t *qo[2];
    int32_t *tf[2];
    uint32_t *far;      // [V] mask of the pairs waiting above T
    int32_t *farl[2];   // far lists (a vertex is on the live one iff far[v] != 0)
    float delta;        // near-far width; 0: plain frontier Bellman-Ford
    int32_t nsrc;
    MsCtrl *c;
};

__global__ void k_mss_fill(float *d, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        d[i] = kMedusaMax;
}

__global__ void k_mss_init(MsArgs a, const int32_t *sources) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    MsCtrl *c = a.c;
    c->q[0] = c->q[1] = 0ull;
    c->cur = 0;
    c->supersteps = 0;
    c->work = 0;
    c->T = a.delta > 0.f ? a.delta : __uint_as_float(kMsInfBits);
    c->fmin = kMsInfBits;
    c->fl = 0;
    c->advance = 0;
    c->nfar[0] = c->nfar[1] = 0u;
    uint32_t n = 0, m = 0;
    for (int i = 0; i < a.nsrc; i++) {
        const int32_t v = sources[i];
        if (a.front[0][v] == 0u) {
            const uint32_t d = (uint32_t)a.outdeg[v];
            if (d > 0) {
                a.qv[0][n] = v;
                a.qo[0][n] = m;
                for (uint32_t t = (m + kTile - 1) / kTile; t <= (m + d - 1) / kTile; t++)
                    a.tf[0][t] = (int32_t)n;
                n++;
                m += d;
            }
        }
        a.front[0][v] |= 1u << i;
        a.dist[(size_t)v * 32 + i] = 0.0f;
    }
    c->q[0] = ((unsigned long long)n << 32) | m;
    c->done = n == 0;
}

// fmn of every lane into c->fmin (distances are non-negative: their float
// bits order like the numbers)
__device__ __forceinline__ void publish_fmin(MsCtrl *c, float fmn) {
    const unsigned m = __reduce_min_sync(0xffffffffu, __float_as_uint(fmn));
    if ((threadIdx.x & 31) == 0 && m < kMsInfBits) atomicMin(&c->fmin, m);
}

// Each warp relaxes kWarpEdges consecutive frontier edges (edge-balanced over
// the queue's scanned out-degrees), one edge at a time for all 32 sources.
// kNF (near-far buckets): an improved pair is marked near (new distance
// below T) or far in the head's 64-bit mask; a pair improved both ways in
// one superstep ends below T, so the commit takes near over far.
template <bool kNF>
__global__ void __launch_bounds__(256) k_mss_push(MsArgs a) {
    MsCtrl *c = a.c;
    if (c->done) return;
    const float T = kNF ? c->T : 0.f;
    float fmn = __uint_as_float(kMsInfBits);  // least far distance this warp set
    const int cur = c->cur;
    const unsigned long long q = c->q[cur];
    const uint32_t n = (uint32_t)(q >> 32), m = (uint32_t)q;
    const int32_t *qv = cur ? a.qv[1] : a.qv[0];
    const uint32_t *qo = cur ? a.qo[1] : a.qo[0];
    const uint32_t *front = cur ? a.front[1] : a.front[0];
    const int32_t *tf = cur ? a.tf[1] : a.tf[0];
    const uint32_t tiles = (m + kTile - 1) / kTile;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t c0 = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * kWarpEdges; c0 < m;
         c0 += warps * kWarpEdges) {
        // owner entry of the chunk's first edge: a binary search over qo
        // within the entries of its merge-path tile (tf[t] holds edge t*kTile,
        // tf[t+1] edge (t+1)*kTile > c0), not over the whole queue
        const uint32_t t = (uint32_t)c0 / kTile;
        int lo = tf[t], hi = t + 1 < tiles ? tf[t + 1] + 1 : (int)n;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (qo[mid] <= (uint32_t)c0) lo = mid; else hi = mid;
        }
        // lane e loads edge c0+e (coalesced): its vertex, weight and owner
        // the chunk's 32 edges span at most 33 entries (every entry has an
        // edge): each lane searches [lo, lo+33)
        const uint32_t my = (uint32_t)c0 + lane;
        int j = lo;
        {
            int l2 = lo, h2 = min((int)n, lo + 33);
            while (h2 - l2 > 1) {
                const int mid = (l2 + h2) >> 1;
                if (qo[mid] <= my) l2 = mid; else h2 = mid;
            }
            j = l2;
        }
        int32_t v = -1, u = -1;
        float w = 0.f;
        if (my < m) {
            u = qv[j];
            const int32_t e = a.row[u] + (int32_t)(my - qo[j]);
            v = __ldg(&a.col[e]);
            w = __ldg(&a.wt[e]);
        }
        int32_t cu = -1;
        uint32_t fm = 0, newly = 0;  // newly: edges whose head this warp touched first
        float du = 0.f;
        for (int k = 0; k < kWarpEdges; k++) {
            const int32_t vk = __shfl_sync(0xffffffffu, v, k);
            if (vk < 0) break;  // warp-uniform: past the last frontier edge
            const int32_t uk = __shfl_sync(0xffffffffu, u, k);
            const float wk = __shfl_sync(0xffffffffu, w, k);
            if (uk != cu) {  // warp-uniform: a new tail vertex
                cu = uk;
                fm = front[uk];
                du = __ldcg(&a.dist[(size_t)uk * 32 + lane]);
            }
            bool imp = false;
            float nd = 0.f;
            if ((fm >> lane) & 1u) {
                nd = du + wk;
                float *pv = &a.dist[(size_t)vk * 32 + lane];
                if (nd < __ldcg(pv)) {
                    atomicMin((unsigned *)pv, __float_as_uint(nd));
                    imp = true;
                    if (kNF && !(nd < T)) fmn = fminf(fmn, nd);
                }
            }
            const uint32_t mask = __ballot_sync(0xffffffffu, imp);
            if (mask) {  // warp-uniform
                if (kNF) {
                    const uint32_t mn = __ballot_sync(0xffffffffu, imp && nd < T);
                    if (lane == 0 &&
                        atomicOr(&a.nxt2[vk], ((unsigned long long)(mask & ~mn) << 32) | mn) == 0ull)
                        newly |= 1u << k;
                } else if (lane == 0 && atomicOr(&a.nxt[vk], mask) == 0u) {
                    newly |= 1u << k;
                }
            }
        }
        // one aggregated append per warp: lane e appends its edge's head
        newly = __shfl_sync(0xffffffffu, newly, 0);
        const bool mine = (newly >> lane) & 1u;
        if (newly) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&c->touched, (uint32_t)__popc(newly));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (mine) a.touched[base + __popc(newly & lanemask_lt())] = v;
        }
    }
    if (kNF) publish_fmin(c, fmn);
}

// Warp-cooperative split of every lane's (vertex v, source mask m): the bits
// of m whose source's distance to v is below T come back, and fmn takes the
// least distance among the other bits.  All 32 lanes call it; lanes with
// m == 0 take no part (their v is not read).  Eight vertices' lines are
// loaded at a time, so their reads overlap.
__device__ __forceinline__ uint32_t split_near(const float *dist, int32_t v, uint32_t m, float T,
                                               float &fmn) {
    const int lane = threadIdx.x & 31;
    uint32_t near = 0u;
    const uint32_t any = __ballot_sync(0xffffffffu, m != 0u);
    for (int k0 = 0; k0 < 32; k0 += 8) {
        if (!((any >> k0) & 0xffu)) continue;  // warp-uniform
        float d[8];
        uint32_t mk[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int32_t vk = __shfl_sync(0xffffffffu, v, k0 + j);
            mk[j] = __shfl_sync(0xffffffffu, m, k0 + j);
            d[j] = mk[j] ? __ldcg(&dist[(size_t)vk * 32 + lane]) : 0.f;  // the vertex's line
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint32_t nm = __ballot_sync(0xffffffffu, d[j] < T) & mk[j];
            if (lane == k0 + j) near = nm;
            if (((mk[j] & ~nm) >> lane) & 1u) fmn = fminf(fmn, d[j]);
        }
    }
    return near;
}

// Warp-aggregated append of the predicated lanes' v to list[*cnt ...].
__device__ __forceinline__ void append_warp(bool pred, int32_t v, uint32_t *cnt, int32_t *list) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(cnt, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) list[base + __popc(mask & lanemask_lt())] = v;
}

// commit: touched vertices take their new masks and join the next queue.
// With near-far buckets (kNF) only their near pairs do; the far ones wait
// in far[v].  A mask is read only by the push over the queue it was
// written for (every queue entry's mask is assigned by this kernel or the
// far pass just before), so old masks are left as they are.
template <bool kNF>
__global__ void k_mss_commit(MsArgs a) {
    MsCtrl *c = a.c;
    if (c->done) return;
    const int nx = c->cur ^ 1;
    const uint32_t nt = c->touched;
    uint32_t *front_nx = nx ? a.front[1] : a.front[0];
    const int fl = kNF ? c->fl : 0;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < nt;
         base += warps * 32) {
        const int64_t i = base + lane;
        bool join = false, wait = false;
        int32_t v = 0;
        uint32_t deg = 0;
        if (i < nt) {
            v = a.touched[i];
            uint32_t near;
            deg = (uint32_t)a.outdeg[v];
            if (kNF) {
                const unsigned long long b = a.nxt2[v];
                a.nxt2[v] = 0ull;
                near = (uint32_t)b;
                const uint32_t fm = (uint32_t)(b >> 32) & ~near;
                // a vertex without out-edges relaxes nothing: no bucket
                if (deg > 0 && fm) wait = atomicOr(&a.far[v], fm) == 0u;  // first: list it
            } else {
                near = a.nxt[v];
                a.nxt[v] = 0u;
            }
            join = deg > 0 && near != 0u;
            if (join) front_nx[v] = near;
        }
        if (kNF) append_warp(wait, v, &c->nfar[fl], fl ? a.farl[1] : a.farl[0]);
        enqueue_warp(join, v, deg, &c->q[nx], nx ? a.qv[1] : a.qv[0], nx ? a.qo[1] : a.qo[0],
                     nx ? a.tf[1] : a.tf[0]);
    }
}

// The queue ran dry with pairs waiting: T becomes fmin + delta and the far
// lists swap.  fmin >= T (recorded under the current threshold) and the
// pair that set it has a distance <= fmin, so the far pass requeues it --
// unless that pair was also improved below T in the same superstep (near
// won, it is not parked).  Then the pass may requeue nothing; it leaves
// fmin exact (the least parked distance), and the next superstep, empty,
// ends in another far pass that does requeue.  (A parked pair whose
// distance dropped later through a near improvement lies below T and is
// simply requeued once more.)
__global__ void k_mss_advance(MsArgs a) {
    MsCtrl *c = a.c;
    if (!c->advance) return;
    const float fm = __uint_as_float(c->fmin);
    float t = fm + a.delta;
    if (fm < __uint_as_float(kMsInfBits) && !(t > fm))
        t = __uint_as_float(c->fmin + 1u);  // the sum rounded back: one float step
    c->T = t;
    c->fmin = kMsInfBits;
    c->fl ^= 1;
    c->nfar[c->fl] = 0u;
}

// The far pass after k_mss_advance: every vertex of the old far list puts
// its pairs now below T into the frontier (front[cur], queue cur); the rest
// stay in far[v] and the vertex moves to the live far list.
__global__ void k_mss_far(MsArgs a) {
    MsCtrl *c = a.c;
    if (!c->advance) return;
    const int fl = c->fl, scan = fl ^ 1, cur = c->cur;
    const uint32_t n = c->nfar[scan];
    const float T = c->T;
    const int32_t *list = scan ? a.farl[1] : a.farl[0];
    uint32_t *front_cur = cur ? a.front[1] : a.front[0];
    float fmn = __uint_as_float(kMsInfBits);
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < n;
         base += warps * 32) {
        const int64_t i = base + lane;
        int32_t v = 0;
        uint32_t m = 0u;
        if (i < n) {
            v = list[i];
            m = a.far[v];
        }
        const uint32_t near = split_near(a.dist, v, m, T, fmn);
        const uint32_t rem = m & ~near;
        if (i < n) {
            a.far[v] = rem;
            if (near) front_cur[v] = near;
        }
        append_warp(rem != 0u, v, &c->nfar[fl], fl ? a.farl[1] : a.farl[0]);
        enqueue_warp(near != 0u, v, near ? (uint32_t)a.outdeg[v] : 0u, &c->q[cur],
                     cur ? a.qv[1] : a.qv[0], cur ? a.qo[1] : a.qo[0], cur ? a.tf[1] : a.tf[0]);
    }
    publish_fmin(c, fmn);
}

// The host queues several supersteps between two reads of the control
// block: once the run is done, every kernel of a superstep returns at once.
__global__ void k_mss_begin(MsArgs a) {
    MsCtrl *c = a.c;
    if (c->done) return;
    c->advance = 0;
    c->touched = 0;
    c->q[c->cur ^ 1] = 0ull;
    c->work += (uint32_t)c->q[c->cur];
}

__global__ void k_mss_end(MsArgs a) {
    MsCtrl *c = a.c;
    if (c->done) return;
    c->q[c->cur] = 0ull;
    c->cur ^= 1;
    c->supersteps++;
    const bool empty = (c->q[c->cur] >> 32) == 0;
    const bool waiting = c->nfar[c->fl] != 0u;
    c->done = empty && !waiting;
    c->advance = empty && waiting;
}

// [V][32] -> out[s*V + v] for the batch's sources (32x32 tiles transposed
// through shared memory, coalesced both ways); stats per source
__global__ void __launch_bounds__(256) k_mss_out(MsArgs a, float *out, unsigned long long *stats) {
    __shared__ float tile[32][33];
    unsigned long long er = 0, vr = 0;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 rows of 32
    for (int64_t v0 = (int64_t)blockIdx.x * 32; v0 < a.V; v0 += (int64_t)gridDim.x * 32) {
        for (int r = ty; r < 32; r += 8) {
            const int64_t v = v0 + r;
            tile[r][tx] = v < a.V ? a.dist[v * 32 + tx] : kMedusaMax;
        }
        __syncthreads();
        for (int sidx = ty; sidx < a.nsrc; sidx += 8) {
            const int64_t v = v0 + tx;
            if (v < a.V) {
                const float d = tile[tx][sidx];
                out[(int64_t)sidx * a.V + v] = d;
                if (d < kMedusaMax) {
                    vr++;
                    er += (uint32_t)a.outdeg[v];
                }
            }
        }
        __syncthreads();
    }
    er = warp_sum(er);
    vr = warp_sum(vr);
    if ((threadIdx.x & 31) == 0 && (er | vr)) {
        atomicAdd(&stats[0], er);
        atomicAdd(&stats[1], vr);
    }
}

}  // namespace

void MsSsspState::ensure(const Graph &g) {
    if (built && V == g.V && E == g.E) return;
    release();
    V = g.V;
    E = g.E;
    const size_t vb = (size_t)V;
    dist.reserve(sizeof(float) * 32 * vb);
    front[0].reserve(4 * vb);
    front[1].reserve(4 * vb);
    nxt.reserve(8 * vb);  // 64-bit masks with near-far buckets
    touched.reserve(4 * vb);
    const size_t tiles = (size_t)(E / kTile) + 2;
    for (int i = 0; i < 2; i++) {
        qv[i].reserve(4 * vb);
        qo[i].reserve(4 * vb);
        tf[i].reserve(4 * tiles);
        farl[i].reserve(4 * vb);
    }
    far.reserve(4 * vb);
    bool bad = false;
    sssp_weight_stats(g, &mean_w, &bad);
    weights_ok = !bad;
    ctrl.reserve(sizeof(MsCtrl));
    stats.reserve(2 * sizeof(unsigned long long));
    srcs.reserve(32 * sizeof(int32_t));
    built = true;
}

float mss_default_delta(const Graph &g, double mean_w) {
    // measured (32 sources, CUDA events): R-MAT 2^20 / 2^24 and 2^22 / 2^26
    // (a = 0.45, weights 1..1000) run fastest at widths 100-200, 1.2-1.45x
    // faster than without buckets; wider ones lose their gain (400: none).
    // With a hub of more than E/1024 out-edges (a = 0.57) every width is
    // slower: the traversal takes 17 supersteps without buckets.  Graphs
    // without hubs want widths from 0.8x (uniform) to 4x (grid) the mean
    // weight, and smaller ones are 1.3-3x slower: they are left to tuning.
    if (g.E == 0 || g.max_outdeg <= 64 || (int64_t)g.max_outdeg > g.E / 1024) return 0.f;
    return (float)std::max(1.0, std::floor(mean_w * 0.3));
}

float mss_delta(const Context &ctx, const Graph &g, const MsSsspState &st) {
    if (!st.weights_ok) return 0.f;
    const int64_t t = ctx.tunable[MB_TUNE_MSS_DELTA];
    if (t >= 0) return (float)t;
    return mss_default_delta(g, st.mean_w);
}

void run_mssssp(Context &ctx, Graph &g, MsSsspState &st, const int32_t *sources, int32_t nsrc,
                float *dist_dev, mb_stats *stats) {
    if (nsrc < 1 || nsrc > 32) fail(MB_ERR_INVALID, "batched SSSP takes 1..32 sources");
    st.ensure(g);
    cudaStream_t s = ctx.stream;
    MsArgs a;
    a.V = g.V;
    a.E = g.E;
    a.row = g.row.as<int32_t>();
    a.col = g.col.as<int32_t>();
    a.outdeg = g.outdeg.as<int32_t>();
    a.wt = g.wt.as<float>();
    a.dist = st.dist.as<float>();
    a.front[0] = st.front[0].as<uint32_t>();
    a.front[1] = st.front[1].as<uint32_t>();
    a.nxt = st.nxt.as<uint32_t>();
    a.nxt2 = st.nxt.as<unsigned long long>();
    a.touched = st.touched.as<int32_t>();
    for (int i = 0; i < 2; i++) {
        a.qv[i] = st.qv[i].as<int32_t>();
        a.qo[i] = st.qo[i].as<uint32_t>();
        a.tf[i] = st.tf[i].as<int32_t>();
    }
    a.far = st.far.as<uint32_t>();
    a.farl[0] = st.farl[0].as<int32_t>();
    a.farl[1] = st.farl[1].as<int32_t>();
    a.delta = mss_delta(ctx, g, st);
    const bool nf = a.delta > 0.f;
    a.nsrc = nsrc;
    a.c = st.ctrl.as<MsCtrl>();
    const size_t vb = (size_t)g.V;
    const int gv = ctx.num_sms * 8;
    MsCtrl *hc = (MsCtrl *)ctx.ctrl_readback();
    cudaEvent_t e0, e1;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    int64_t launches = 0;
    try {
        MB_CUDA(cudaMemcpyAsync(st.srcs.p, sources, sizeof(int32_t) * nsrc, cudaMemcpyHostToDevice, s));
        MB_CUDA(cudaEventRecord(e0, s));
        k_mss_fill<<<gv, 256, 0, s>>>(a.dist, (int64_t)vb * 32);
        MB_CUDA(cudaMemsetAsync(a.front[0], 0, 4 * vb, s));
        MB_CUDA(cudaMemsetAsync(a.front[1], 0, 4 * vb, s));
        MB_CUDA(cudaMemsetAsync(a.nxt, 0, (nf ? 8 : 4) * vb, s));
        if (nf) MB_CUDA(cudaMemsetAsync(a.far, 0, 4 * vb, s));
        MB_CUDA(cudaMemsetAsync(st.stats.p, 0, 2 * sizeof(unsigned long long), s));
        k_mss_init<<<1, 32, 0, s>>>(a, st.srcs.as<int32_t>());
        launches += 2;
        MB_CHECK_LAUNCH();
        // every superstep lowers some distance; integer distances below 2^24
        // bound the count well below this cap.  With buckets a bucket may
        // advance a single (vertex, source) pair, so the cap scales with the
        // sources.
        const int64_t cap = step_cap(ctx, ((int64_t)g.V * 4 + 16) * (nf ? nsrc : 1));
        // the control block is read after the first superstep and then after
        // every kSupersteps queued ones (the kernels of a superstep queued
        // past the last one return at once)
        constexpr int kSupersteps = 4;
        for (int64_t it = 0;;) {
            MB_CUDA(cudaMemcpyAsync(hc, a.c, sizeof(MsCtrl), cudaMemcpyDeviceToHost, s));
            MB_CUDA(cudaStreamSynchronize(s));
            if (hc->done) break;
            if (it > cap) fail(MB_ERR_TIMEOUT, "batched sssp: superstep cap reached");
            const int batch = it == 0 ? 1 : kSupersteps;
            for (int b = 0; b < batch; b++, it++) {
                if (nf) {  // refill the queue from the far pairs when it ran dry
                    k_mss_advance<<<1, 1, 0, s>>>(a);
                    k_mss_far<<<gv, 256, 0, s>>>(a);
                    launches += 2;
                }
                k_mss_begin<<<1, 1, 0, s>>>(a);
                if (nf) {
                    k_mss_push<true><<<gv, 256, 0, s>>>(a);
                    k_mss_commit<true><<<gv, 256, 0, s>>>(a);
                } else {
                    k_mss_push<false><<<gv, 256, 0, s>>>(a);
                    k_mss_commit<false><<<gv, 256, 0, s>>>(a);
                }
                k_mss_end<<<1, 1, 0, s>>>(a);
                launches += 4;
                MB_CHECK_LAUNCH();
            }
        }
        k_mss_out<<<gv, 256, 0, s>>>(a, dist_dev, st.stats.as<unsigned long long>());
        launches++;
        MB_CHECK_LAUNCH();
        MB_CUDA(cudaEventRecord(e1, s));
        MB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        MB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        unsigned long long hs[2];
        MB_CUDA(cudaMemcpy(hs, st.stats.p, sizeof(hs), cudaMemcpyDeviceToHost));
        if (stats) {
            *stats = mb_stats{};
            stats->supersteps = hc->supersteps;
            stats->edges_traversed = (int64_t)hs[0];
            stats->vertices_reached = (int64_t)hs[1];
            stats->device_ms = ms;
            stats->schedule_count[MB_SCHED_PUSH_EDGE_QUEUE] = hc->supersteps;
            stats->kernel_launches = launches;
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
