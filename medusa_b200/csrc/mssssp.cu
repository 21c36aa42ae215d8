// mssssp.cu -- batched SSSP: up to 32 sources in one traversal.
//
// Distances are stored vertex-major, dist[v*32 + s], so the 32 distances of a
// vertex fill one 128-byte line.  front[v] is the 32-bit mask of the sources
// whose distance to v dropped in the last superstep.  A warp relaxes one edge
// (u,v,w) for every source at once -- lane s holds source s -- so reading
// and updating dist[v][*] is one coalesced line; the lanes that improved are
// combined with __ballot_sync into v's mask of the next frontier.
// Per source this is the same frontier Bellman-Ford as mb_sssp (integer-
// valued float distances, exact minima), so dist_out[s*V + v] equals 32
// single-source runs bit for bit.  No reference counterpart exists for the
// batching itself.
#include <algorithm>
#include "mssssp.cuh"

namespace mb {
namespace {

constexpr int kWarpEdges = 32;  // consecutive edges a warp relaxes per pass

struct MsCtrl {
    unsigned long long q[2];
    uint32_t touched;
    int32_t cur;
    int32_t supersteps;
    int32_t done;
    unsigned long long work;  // edges relaxed (for all sources of a batch)
};

struct MsArgs {
    int32_t V;
    int64_t E;
    const int32_t *row, *col, *outdeg;
    const float *wt;
    float *dist;  // [V][32]
    uint32_t *front[2], *nxt;
    int32_t *touched;
    int32_t *qv[2];
    uint32_t *qo[2];
    int32_t *tf[2];
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

// Each warp relaxes kWarpEdges consecutive frontier edges (edge-balanced over
// the queue's scanned out-degrees), one edge at a time for all 32 sources.
__global__ void __launch_bounds__(256) k_mss_push(MsArgs a) {
    MsCtrl *c = a.c;
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
            if ((fm >> lane) & 1u) {
                const float nd = du + wk;
                float *pv = &a.dist[(size_t)vk * 32 + lane];
                if (nd < __ldcg(pv)) {
                    atomicMin((unsigned *)pv, __float_as_uint(nd));
                    imp = true;
                }
            }
            const uint32_t mask = __ballot_sync(0xffffffffu, imp);
            if (mask && lane == 0 && atomicOr(&a.nxt[vk], mask) == 0u) newly |= 1u << k;
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
}

// commit: clear the old frontier masks; touched vertices take their new
// masks and join the next queue
__global__ void k_mss_commit(MsArgs a) {
    MsCtrl *c = a.c;
    const int cur = c->cur, nx = cur ^ 1;
    const uint32_t nold = (uint32_t)(c->q[cur] >> 32), nt = c->touched;
    uint32_t *front_cur = cur ? a.front[1] : a.front[0];
    uint32_t *front_nx = cur ? a.front[0] : a.front[1];
    const int32_t *qv = cur ? a.qv[1] : a.qv[0];
    const int lane = threadIdx.x & 31;
    const int64_t total = (int64_t)nold + nt;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < total;
         base += warps * 32) {
        const int64_t i = base + lane;
        bool join = false;
        int32_t v = 0;
        uint32_t deg = 0;
        if (i < nold) {
            front_cur[qv[i]] = 0u;
        } else if (i < total) {
            v = a.touched[i - nold];
            const uint32_t nb = a.nxt[v];
            a.nxt[v] = 0u;
            front_nx[v] = nb;
            deg = (uint32_t)a.outdeg[v];
            join = deg > 0;
        }
        enqueue_warp(join, v, deg, &c->q[nx], nx ? a.qv[1] : a.qv[0], nx ? a.qo[1] : a.qo[0],
                     nx ? a.tf[1] : a.tf[0]);
    }
}

__global__ void k_mss_begin(MsArgs a) {
    MsCtrl *c = a.c;
    c->touched = 0;
    c->q[c->cur ^ 1] = 0ull;
    c->work += (uint32_t)c->q[c->cur];
}

__global__ void k_mss_end(MsArgs a) {
    MsCtrl *c = a.c;
    c->q[c->cur] = 0ull;
    c->cur ^= 1;
    c->supersteps++;
    c->done = (c->q[c->cur] >> 32) == 0;
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
    nxt.reserve(4 * vb);
    touched.reserve(4 * vb);
    const size_t tiles = (size_t)(E / kTile) + 2;
    for (int i = 0; i < 2; i++) {
        qv[i].reserve(4 * vb);
        qo[i].reserve(4 * vb);
        tf[i].reserve(4 * tiles);
    }
    ctrl.reserve(sizeof(MsCtrl));
    stats.reserve(2 * sizeof(unsigned long long));
    srcs.reserve(32 * sizeof(int32_t));
    built = true;
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
    a.touched = st.touched.as<int32_t>();
    for (int i = 0; i < 2; i++) {
        a.qv[i] = st.qv[i].as<int32_t>();
        a.qo[i] = st.qo[i].as<uint32_t>();
        a.tf[i] = st.tf[i].as<int32_t>();
    }
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
        MB_CUDA(cudaMemsetAsync(a.nxt, 0, 4 * vb, s));
        MB_CUDA(cudaMemsetAsync(st.stats.p, 0, 2 * sizeof(unsigned long long), s));
        k_mss_init<<<1, 32, 0, s>>>(a, st.srcs.as<int32_t>());
        launches += 2;
        MB_CHECK_LAUNCH();
        // every superstep lowers some distance; integer distances below 2^24
        // bound the count well below this cap
        const int64_t cap = step_cap(ctx, (int64_t)g.V * 4 + 16);
        for (int64_t it = 0;; it++) {
            MB_CUDA(cudaMemcpyAsync(hc, a.c, sizeof(MsCtrl), cudaMemcpyDeviceToHost, s));
            MB_CUDA(cudaStreamSynchronize(s));
            if (hc->done) break;
            if (it > cap) fail(MB_ERR_TIMEOUT, "batched sssp: superstep cap reached");
            k_mss_begin<<<1, 1, 0, s>>>(a);
            k_mss_push<<<gv, 256, 0, s>>>(a);
            k_mss_commit<<<gv, 256, 0, s>>>(a);
            k_mss_end<<<1, 1, 0, s>>>(a);
            launches += 4;
            MB_CHECK_LAUNCH();
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
