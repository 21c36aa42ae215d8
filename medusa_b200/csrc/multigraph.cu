// multigraph.cu -- many independent graphs of uneven sizes in ONE persistent
// launch, fed by a device-side work queue.
//
// Each graph g gets a team of T_g CTAs, T_g growing with its edge count (the
// edges per CTA and the CTA size are tunables the autotuner sets).  The work
// queue is a list of (graph, member) entries, largest graph first, handed
// out by one atomic counter; a CTA that takes an entry runs its share of the
// graph -- `pr_iters` PageRank supersteps, then one BFS -- and synchronises
// with its team mates through a barrier in the graph's team state.  The
// launch is cooperative, so every CTA is resident: entries are handed out
// in order and a team's entries are consecutive, so at most one team is
// ever incomplete and the CTAs of complete teams always come back for more
// -- every barrier wait ends.  Every wait is also bounded: past kTeamSpins
// polls the CTA sets the batch's error flag and every CTA leaves.
//
// PageRank follows the fixed summation order of pr_order.cuh, so each
// graph's ranks equal mb_pagerank's on that graph bit for bit.  The BFS is
// level-synchronous and direction-optimising per level (top-down from the
// queue while the frontier holds fewer than V/20 vertices, else bottom-up),
// which gives the reference's levels (Algorithm/CPUFunctorHoster.cpp:16-65).
// No reference counterpart exists for the batching itself.
#include <algorithm>
#include <cmath>
#include "frontier.cuh"
#include "multigraph.cuh"
#include "pr_order.cuh"

namespace mb {
void graph_generate(Context &ctx, Graph &g, const mb_gen_params &p, uint32_t flags);

namespace {

constexpr long kTeamSpins = 1l << 24;  // polls (64 ns apart) before a barrier gives up (default)

struct MultiArgs {
    const GDesc *desc;
    TeamState *team;
    const int2 *entries;  // (graph, member), largest graph first
    int32_t nentries;
    int32_t pr_iters;
    float *contrib[2];    // batch-wide, graph g at desc[g].vbase
    int32_t *queue[2];
    float *rank;          // outputs, batch-wide
    int32_t *level;
    unsigned *work;       // [0] next entry, [1] error flag, [2] launches
    long wait_polls;      // polls before a team barrier gives up
};

// Team barrier (all threads of the CTA call it).  False if it gave up or
// another CTA reported an error.
__device__ bool team_sync(TeamState *ts, int t, unsigned *err, long polls) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        if (t > 1) {
            const unsigned gen = __ldcg(&ts->bar_gen);
            const unsigned arrived = atomicAdd(&ts->bar_count, 1u);
            if (arrived == (unsigned)t - 1) {
                atomicExch(&ts->bar_count, 0u);
                __threadfence();
                atomicAdd(&ts->bar_gen, 1u);
            } else {
                ok = 0;
                for (long it = 0; it < polls; it++) {
                    if (__ldcg(&ts->bar_gen) != gen) {
                        ok = 1;
                        break;
                    }
                    if (__ldcg(err)) break;
                    __nanosleep(64);
                }
                if (!ok) atomicExch(err, 1u);
            }
            __threadfence();
        }
        s_ok = ok && !__ldcg(err);
    }
    __syncthreads();
    return s_ok;
}

// Append v (where pred) to the team's next queue; all lanes call it.
__device__ __forceinline__ void append_warp(bool pred, int32_t v, unsigned *count, int32_t *q) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) q[base + __popc(mask & lanemask_lt())] = v;
}

struct Member {
    int k, t;             // member index, team size
    int64_t tid, nthr;    // thread index and count across the team
    int64_t warp, nwarp;  // warp index and count across the team
};

__device__ bool pr_phase(const MultiArgs &a, const GDesc &d, TeamState *ts, const Member &m) {
    const float init = 1.0f / (float)d.V;
    float *c0 = a.contrib[0] + d.vbase, *c1 = a.contrib[1] + d.vbase;
    float *rank = a.rank + d.vbase;
    for (int64_t v = m.tid; v < d.V; v += m.nthr) {
        const int32_t deg = d.row[v + 1] - d.row[v];
        c0[v] = deg > 0 ? init / (float)deg : 0.0f;
        if (a.pr_iters == 0) rank[v] = init;
    }
    if (!team_sync(ts, m.t, &a.work[1], a.wait_polls)) return false;
    const int lane = threadIdx.x & 31;
    const int64_t ngroups = ((int64_t)d.V + 31) / 32;
    for (int it = 0; it < a.pr_iters; it++) {
        const float *cin = (it & 1) ? c1 : c0;
        float *cout = (it & 1) ? c0 : c1;
        for (int64_t grp = m.warp; grp < ngroups; grp += m.nwarp) {
            const int32_t v = (int32_t)(grp * 32 + lane);
            const bool valid = v < d.V;
            int32_t b = 0, e = 0;
            if (valid) {
                b = __ldg(&d.rrow[v]);
                e = __ldg(&d.rrow[v + 1]);
            }
            const bool heavy = valid && (e - b) > kPrLight;
            float sum = 0.f;
            if (valid && !heavy) {
#pragma unroll 4
                for (int32_t j = b; j < e; j++) sum += __ldcg(&cin[__ldg(&d.rcol[j])]);
            }
            for (unsigned hm = __ballot_sync(0xffffffffu, heavy); hm; hm &= hm - 1) {
                const int owner = __ffs(hm) - 1;
                const int32_t hb = __shfl_sync(0xffffffffu, b, owner);
                const int32_t he = __shfl_sync(0xffffffffu, e, owner);
                float tot = 0.f;
                for (int64_t j0 = hb; j0 < he; j0 += kPrBlock) {
                    const int64_t j1 = min((int64_t)he, j0 + kPrBlock);
                    tot += pr_warp_block_sum(j0, j1, [&](int64_t j) { return __ldcg(&cin[__ldg(&d.rcol[j])]); });
                }
                if (lane == owner) sum = tot;
            }
            if (valid) {
                const float r = pr_update(sum);
                rank[v] = r;
                const int32_t deg = __ldg(&d.row[v + 1]) - __ldg(&d.row[v]);
                cout[v] = deg > 0 ? r / (float)deg : 0.0f;
            }
        }
        if (!team_sync(ts, m.t, &a.work[1], a.wait_polls)) return false;
    }
    return true;
}

__device__ bool bfs_phase(const MultiArgs &a, const GDesc &d, TeamState *ts, const Member &m) {
    int32_t *lv = a.level + d.vbase;
    int32_t *q[2] = {a.queue[0] + d.vbase, a.queue[1] + d.vbase};
    for (int64_t v = m.tid; v < d.V; v += m.nthr) lv[v] = -1;
    if (!team_sync(ts, m.t, &a.work[1], a.wait_polls)) return false;
    if (m.k == 0 && threadIdx.x == 0) {
        lv[d.source] = 0;
        q[0][0] = d.source;
        ts->qn[0] = 1;
    }
    if (!team_sync(ts, m.t, &a.work[1], a.wait_polls)) return false;
    const int lane = threadIdx.x & 31;
    for (int32_t L = 0;; L++) {
        const int cur = L % 3, nxt = (L + 1) % 3, clr = (L + 2) % 3;
        const unsigned n = __ldcg(&ts->qn[cur]);
        if (n == 0) break;  // every member reads the same count
        // the counter of level L-1 is read by nobody any more
        if (m.k == 0 && threadIdx.x == 0) ts->qn[clr] = 0;
        const int32_t *qc = q[L & 1];
        int32_t *qx = q[(L + 1) & 1];
        unsigned *cnt = &ts->qn[nxt];
        if ((int64_t)n * 20 > (int64_t)d.V) {
            // bottom-up: each unvisited vertex looks for a parent at level L
            for (int64_t base = m.warp * 32; base < d.V; base += m.nwarp * 32) {
                const int32_t v = (int32_t)(base + lane);
                bool found = false;
                if (v < d.V && __ldcg(&lv[v]) == -1) {
                    const int32_t jb = __ldg(&d.rrow[v]), je = __ldg(&d.rrow[v + 1]);
                    for (int32_t j = jb; j < je; j++) {
                        if (__ldcg(&lv[__ldg(&d.rcol[j])]) == L) {
                            found = true;
                            break;
                        }
                    }
                    if (found) lv[v] = L + 1;
                }
                append_warp(found, v, cnt, qx);
            }
        } else {
            // top-down from the queue: warps for lists of 32 or more, lanes below
            auto visit = [&](bool valid, int32_t v) {
                const bool claim = valid && __ldcg(&lv[v]) == -1 && atomicCAS(&lv[v], -1, L + 1) == -1;
                append_warp(claim, v, cnt, qx);
            };
            for (int64_t base = m.warp * 32; base < n; base += m.nwarp * 32) {
                const int64_t i = base + lane;
                int32_t st = 0, deg = 0;
                if (i < n) {
                    const int32_t u = __ldcg(&qc[i]);
                    st = __ldg(&d.row[u]);
                    deg = __ldg(&d.row[u + 1]) - st;
                }
                for (unsigned big = __ballot_sync(0xffffffffu, deg >= 32); big; big &= big - 1) {
                    const int l = __ffs(big) - 1;
                    const int32_t bst = __shfl_sync(0xffffffffu, st, l);
                    const int32_t bdeg = __shfl_sync(0xffffffffu, deg, l);
                    for (int32_t k = 0; k < bdeg; k += 32)
                        visit(k + lane < bdeg, k + lane < bdeg ? __ldg(&d.col[bst + k + lane]) : 0);
                }
                const int32_t sd = deg < 32 ? deg : 0;
                int32_t maxd = sd;
#pragma unroll
                for (int off = 16; off; off >>= 1) maxd = max(maxd, __shfl_xor_sync(0xffffffffu, maxd, off));
                for (int32_t r = 0; r < maxd; r++) visit(r < sd, r < sd ? __ldg(&d.col[st + r]) : 0);
            }
        }
        if (!team_sync(ts, m.t, &a.work[1], a.wait_polls)) return false;
    }
    // reached vertices and their out-edges (the traversal count)
    unsigned long long nr = 0, er = 0;
    for (int64_t v = m.tid; v < d.V; v += m.nthr) {
        if (__ldcg(&lv[v]) >= 0) {
            nr++;
            er += (unsigned)(__ldg(&d.row[v + 1]) - __ldg(&d.row[v]));
        }
    }
    nr = warp_sum(nr);
    er = warp_sum(er);
    if (lane == 0 && nr) {
        atomicAdd(&ts->reached, nr);
        atomicAdd(&ts->reached_edges, er);
    }
    return true;
}

__global__ void k_multi(MultiArgs a) {
    __shared__ int s_e;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.work[2], 1u);
    const int wpc = blockDim.x >> 5;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_e = (int)atomicAdd(&a.work[0], 1u);
        __syncthreads();
        const int e = s_e;
        if (e >= a.nentries || __ldcg(&a.work[1])) break;
        const int2 en = a.entries[e];
        const GDesc d = a.desc[en.x];
        TeamState *ts = &a.team[en.x];
        Member m;
        m.k = en.y;
        m.t = d.team;
        m.tid = (int64_t)m.k * blockDim.x + threadIdx.x;
        m.nthr = (int64_t)m.t * blockDim.x;
        m.warp = (int64_t)m.k * wpc + (threadIdx.x >> 5);
        m.nwarp = (int64_t)m.t * wpc;
        if (!pr_phase(a, d, ts, m)) continue;  // the error flag ends the loop
        bfs_phase(a, d, ts, m);
    }
}

}  // namespace

// Keep the CSR and the reverse CSR of graph i (all the batch kernel reads)
// and count it into the batch's vertex offsets.
static void batch_take(Batch &b, int32_t i) {
    b.graphs[i].esrc.release();
    b.graphs[i].wt.release();
    b.graphs[i].rwt.release();
    b.graphs[i].mslot.release();
    b.vbase.push_back(b.vbase.back() + b.graphs[i].V);
    b.total_E += b.graphs[i].E;
}

void batch_generate(Context &ctx, Batch &b, const mb_gen_params *params, int32_t n) {
    b.release();
    b.graphs.resize(n);
    b.vbase.assign(1, 0);
    for (int32_t i = 0; i < n; i++) {
        graph_generate(ctx, b.graphs[i], params[i], MB_ORDER_REFERENCE);
        batch_take(b, i);
    }
    batch_finish(b);
}

void batch_from_edges(Context &ctx, Batch &b, int32_t n, const int32_t *nv, const int64_t *ne,
                      const int32_t *src, const int32_t *dst) {
    b.release();
    b.graphs.resize(n);
    b.vbase.assign(1, 0);
    int64_t e0 = 0;
    for (int32_t i = 0; i < n; i++) {
        DevBuf bs, bd;
        try {
            const size_t eb = sizeof(uint32_t) * (size_t)std::max<int64_t>(ne[i], 1);
            bs.reserve(eb);
            bd.reserve(eb);
            copy_sync(ctx.stream, bs.p, src + e0, 4 * (size_t)ne[i]);
            copy_sync(ctx.stream, bd.p, dst + e0, 4 * (size_t)ne[i]);
            graph_build_from_device_edges(ctx, b.graphs[i], nv[i], ne[i], bs.as<uint32_t>(),
                                          bd.as<uint32_t>(), nullptr, MB_ORDER_REFERENCE);
        } catch (...) {
            bs.release();
            bd.release();
            throw;
        }
        bs.release();
        bd.release();
        batch_take(b, i);
        e0 += ne[i];
    }
    batch_finish(b);
}

void batch_finish(Batch &b) {
    const int32_t n = (int32_t)b.graphs.size();
    b.total_V = b.vbase.back();
    const size_t vb = (size_t)std::max<int64_t>(b.total_V, 1);
    for (int i = 0; i < 2; i++) {
        b.contrib[i].reserve(sizeof(float) * vb);
        b.queue[i].reserve(sizeof(int32_t) * vb);
    }
    b.desc.reserve(sizeof(GDesc) * std::max(n, 1));
    b.team.reserve(sizeof(TeamState) * std::max(n, 1));
    b.work.reserve(4 * sizeof(unsigned));
    b.desc_gen = -1;
}

void batch_run(Context &ctx, Batch &b, int32_t pr_iters, const int32_t *sources, float *ranks_dev,
               int32_t *levels_dev, mb_stats *stats) {
    const int32_t n = (int32_t)b.graphs.size();
    cudaStream_t s = ctx.stream;
    const int threads = (int)(ctx.tunable[MB_TUNE_BATCH_THREADS] > 0 ? ctx.tunable[MB_TUNE_BATCH_THREADS] : 256);
    const int64_t epc = ctx.tunable[MB_TUNE_BATCH_EDGES_PER_CTA] > 0 ? ctx.tunable[MB_TUNE_BATCH_EDGES_PER_CTA]
                                                                     : (int64_t)1 << 16;
    int per_sm = 0;
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_multi, threads, 0));
    if (per_sm < 1) fail(MB_ERR_UNSUPPORTED, "batch kernel does not fit on an SM");
    const int grid = ctx.num_sms * per_sm;
    // descriptors and the work queue (largest graph first)
    std::vector<GDesc> desc(n);
    std::vector<int32_t> order(n);
    int64_t nent = 0;
    for (int32_t i = 0; i < n; i++) {
        const Graph &g = b.graphs[i];
        GDesc &d = desc[i];
        d.V = g.V;
        d.E = (int32_t)g.E;
        d.row = g.row.as<int32_t>();
        d.col = g.col.as<int32_t>();
        d.rrow = g.rrow.as<int32_t>();
        d.rcol = g.rcol.as<int32_t>();
        d.vbase = b.vbase[i];
        d.team = (int32_t)std::min<int64_t>(std::max<int64_t>(1, (g.E + g.V + epc - 1) / epc), grid);
        d.source = sources ? sources[i] : 0;
        if (d.source < 0 || d.source >= g.V) fail(MB_ERR_INVALID, "batch: source vertex out of range");
        order[i] = i;
        nent += d.team;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return desc[x].E + desc[x].V > desc[y].E + desc[y].V; });
    std::vector<int2> ent;
    ent.reserve((size_t)nent);
    for (int32_t i : order)
        for (int32_t k = 0; k < desc[i].team; k++) ent.push_back(make_int2(i, k));
    b.entries.reserve(sizeof(int2) * std::max<size_t>(ent.size(), 1));
    b.nentries = (int32_t)ent.size();
    MB_CUDA(cudaMemcpyAsync(b.desc.p, desc.data(), sizeof(GDesc) * n, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(b.entries.p, ent.data(), sizeof(int2) * ent.size(), cudaMemcpyHostToDevice, s));
    MultiArgs a;
    a.desc = b.desc.as<GDesc>();
    a.team = b.team.as<TeamState>();
    a.entries = b.entries.as<int2>();
    a.nentries = b.nentries;
    a.pr_iters = pr_iters;
    a.contrib[0] = b.contrib[0].as<float>();
    a.contrib[1] = b.contrib[1].as<float>();
    a.queue[0] = b.queue[0].as<int32_t>();
    a.queue[1] = b.queue[1].as<int32_t>();
    a.rank = ranks_dev;
    a.level = levels_dev;
    a.work = b.work.as<unsigned>();
    a.wait_polls = ctx.tunable[MB_TUNE_WAIT_POLLS] >= 0 ? (long)ctx.tunable[MB_TUNE_WAIT_POLLS] : kTeamSpins;
    cudaEvent_t e0, e1;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    try {
        MB_CUDA(cudaEventRecord(e0, s));
        MB_CUDA(cudaMemsetAsync(b.team.p, 0, sizeof(TeamState) * n, s));
        MB_CUDA(cudaMemsetAsync(b.work.p, 0, 4 * sizeof(unsigned), s));
        void *params[] = {(void *)&a};
        MB_CUDA(cudaLaunchCooperativeKernel((const void *)k_multi, dim3(grid), dim3(threads), params, 0, s));
        MB_CUDA(cudaEventRecord(e1, s));
        MB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        MB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        unsigned work[4];
        MB_CUDA(cudaMemcpy(work, b.work.p, sizeof(work), cudaMemcpyDeviceToHost));
        if (work[1]) fail(MB_ERR_TIMEOUT, "batch: a team barrier timed out");
        std::vector<TeamState> ts(n);
        MB_CUDA(cudaMemcpy(ts.data(), b.team.p, sizeof(TeamState) * n, cudaMemcpyDeviceToHost));
        if (stats) {
            *stats = mb_stats{};
            int64_t reached = 0, redges = 0;
            for (const auto &t : ts) {
                reached += (int64_t)t.reached;
                redges += (int64_t)t.reached_edges;
            }
            stats->supersteps = pr_iters;
            stats->edges_traversed = (int64_t)pr_iters * b.total_E + redges;
            stats->vertices_reached = reached;
            stats->device_ms = ms;
            stats->kernel_launches = work[2];
            stats->edges_scanned = redges;
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
