// sssp_async.cuh -- the asynchronous SSSP kernel (k_sssp_async) and its hub
// chunk tables.  Included by sssp.cu inside its anonymous namespace: it uses
// that file's SsspArgs, ld_dist and the engine's control block.
#pragma once

// ---- asynchronous SSSP (kBranchAsync) ---------------------------------------
// The rest of the traversal, from the current queue frontier to the
// fixpoint (never entered with near-far buckets on: their far pile is not
// part of that frontier), in ONE cooperative launch with no superstep
// barriers: a chaotic
// relaxation ordered by a distance threshold, in the manner of Meyer &
// Sanders' delta-stepping (J. Algorithms 49, 2003) run asynchronously.
//  - a.adirty is the dirty bitmap: v's bit is set when dist[v] dropped and
//    v's out-edges have not yet been relaxed from the new distance;
//  - hubs: a vertex with more than kAsyncChunk out-edges owns one extra id
//    per kAsyncChunk of them.  Chunk c (hub_cbase[v] + j for the j-th of v)
//    sits at id V + (c % 32) * nc32 + c / 32, so the consecutive chunks of a
//    hub fall in different bitmap words and thus to different owner warps.
//    Claiming the hub sets its chunks' bits instead of relaxing; each chunk
//    is then claimed (when the hub's distance is below T) and relaxed by its
//    owner from the hub's distance read at that claim, so one hub's edges
//    spread over many warps and no warp gets a long serial batch;
//  - warp g owns the bitmap words g, g + G, g + 2G, ... (G = warps of the
//    grid; interleaved, so the low-numbered hubs of R-MAT graphs spread out)
//    and scans them: it claims the bits of vertices whose distance is below
//    the threshold T with one atomicAnd per word, re-reads their distances
//    and relaxes their out-edges warp-wide, 32 edges per strip; a lower
//    distance is atomicMin'ed and the neighbour's bit set.  A warp that
//    itself set the bit of a vertex below T claims it back and relaxes it
//    next (local continuation).  A claim is an atomicAnd that returned the
//    bit set, so every set bit has exactly one claimer;
//  - termination: AsyncState::p counts the bits a warp may set (added, and
//    its return awaited, before the warp sets any) and AsyncState::d the
//    part it did not set plus every finished claim.  Both only grow, and
//    sum(p) - sum(d) is never below the bits set plus the claims in flight.
//    A warp reads every d, then every p: equal sums mean that at a moment
//    between the two reads no bit was set and no claim in flight, and from
//    then on nothing can set one, so every warp leaves;
//  - a warp that finds nothing below T reports itself idle once per phase
//    (the CTA's warps in shared memory, then one global count per CTA); the
//    last CTA raises T by delta (or to the least distance seen above T plus
//    delta) and opens the next phase.  T only orders the claims: every order
//    reaches the same fixpoint, the exact distances;
//  - every wait is bounded: the start barrier and a warp's run of idle
//    passes give up after wait_polls (default kAsyncSpins), set ERR_ASYNC
//    and make every warp leave; a warp with more claiming passes than the
//    run's superstep cap sets ERR_STEP_CAP and does the same;
//  - polling: only warp 0 of each CTA reads the termination counters and
//    the abort flag (after an idle pass), and tells its CTA through shared
//    memory; idle warps sleep 128 ns to 2 us between passes.
// Ordering: a value returned by an atomic is used in the operand of the next
// atomic that must come after it (an always-zero shift), so the hardware
// issues the second only once the first has been performed at L2.
constexpr int kAsyncThreads = 256;
constexpr int kAsyncWarps = kAsyncThreads / 32;
#ifndef MB_ASYNC_U
#define MB_ASYNC_U 2
#endif
#ifndef MB_ASYNC_SLEEP_MAX
#define MB_ASYNC_SLEEP_MAX 4  // idle sleep 128 ns << min(idle passes, this)
#endif
constexpr int kAsyncU = MB_ASYNC_U;  // strips of 32 edges in flight per warp
constexpr long kAsyncSpins = 1l << 22;
constexpr uint32_t kInfBits = 0x7f800000u;
static_assert(kAsyncSlots == 32, "one work counter slot per lane");

__device__ __forceinline__ unsigned long long ld_rlx64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ld_rlx32(const void *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t atom_and_acquire(uint32_t *p, uint32_t m) {
    uint32_t old;
    asm volatile("atom.acquire.gpu.global.and.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(m) : "memory");
    return old;
}
__device__ __forceinline__ float warp_min_f(float x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x = fminf(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}
__device__ __forceinline__ void async_abort(Ctrl *c, AsyncState *S, int err) {
    atomicOr(&c->err, err);
    atomicExch((unsigned *)&S->abort_.v, 1u);
}

// True (in every lane) when no dirty bit is set and no claim is in flight.
__device__ __forceinline__ bool async_finished(AsyncState *S) {
    const int lane = threadIdx.x & 31;
    const unsigned long long d = warp_sum(ld_rlx64(&S->d[lane].v));
    // the p loads wait for every d load (d < 2^63: the offset is zero)
    const unsigned long long p = warp_sum(ld_rlx64(&S->p[lane].v + (d >> 63)));
    return p == d;
}

#ifndef MB_ASYNC_CHUNK
#define MB_ASYNC_CHUNK 64
#endif
constexpr int32_t kAsyncChunk = MB_ASYNC_CHUNK;
// Default threshold step of the asynchronous BFS, in hops: 8 measured best
// on the 1448^2 grid (1 -> 94 phases, 1.53 ms; 4 -> 25 phases, 0.85 ms; 8 ->
// 13 phases, 0.73 ms; every vertex still relaxed once).
constexpr float kBfsAsyncDelta = 8.f;
// Relax what this warp claimed: lane l holds one dirty id (or v < 0) -- a
// vertex (its out-edges), a hub (the bits of its chunks) or a chunk (its
// out-edges).  Every item (an edge, or a chunk bit) may set one dirty bit.
// Returns the edges relaxed (every lane).
// Local continuation (MB_ASYNC_LOCAL): a vertex this warp newly makes dirty
// with a distance below the threshold T is also recorded in `nxt` (up to
// kAsyncNext, *nn of them, warp-uniform), and the warp claims and relaxes it
// next itself instead of leaving it to its owner's next pass.
#ifndef MB_ASYNC_LOCAL
#define MB_ASYNC_LOCAL 1
#endif
constexpr uint32_t kAsyncNext = 64;

template <bool kUnit>
__device__ __forceinline__ uint32_t async_relax(const SsspArgs &a, AsyncState *S, int slot, int32_t v,
                                                float T, int32_t *nxt, uint32_t *nn) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    uint32_t *dirty = a.adirty;
    const int32_t V = a.f.V;
    const bool mine = v >= 0;
    const uint32_t claimed = __ballot_sync(FULL, mine);
    int32_t base = 0;   // edge (or chunk id) of the lane's first item
    uint32_t deg = 0;   // its items
    bool hub = false;
    float du = 0.f;
    if (mine) {
        // after the claim (acquire): the latest distances
        if (v < V) {
            const int32_t rs = __ldg(&a.row[v]);
            deg = (uint32_t)(__ldg(&a.row[v + 1]) - rs);
            du = ld_dist(a, v);
            base = rs;
            if (deg > (uint32_t)kAsyncChunk) {
                hub = true;
                base = V + __ldg(&a.hub_cbase[v]);
                deg = (deg + kAsyncChunk - 1) / kAsyncChunk;
            }
        } else {
            const int32_t h = __ldg(&a.chunk_src[v - V]);
            base = __ldg(&a.chunk_rs[v - V]);
            deg = (uint32_t)min(kAsyncChunk, __ldg(&a.row[h + 1]) - base);
            du = ld_dist(a, h);
        }
    }
    const uint32_t incl = warp_incl_scan_u32(deg);
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    const int32_t base_e = base - (int32_t)(incl - deg);  // item k of the owner: base_e(owner) + k
    const uint32_t hubs = __ballot_sync(FULL, hub);
    unsigned long long pre = 0;
    if (lane == 0 && total) pre = atomicAdd(&S->p[slot].v, (unsigned long long)total);
    const int32_t order = (int32_t)(__shfl_sync(FULL, pre, 0) >> 63);  // zero
    uint32_t newly = 0;
    for (uint32_t b0 = 0; b0 < total; b0 += 32 * kAsyncU) {
        int32_t x[kAsyncU];
        float nd[kAsyncU], dx[kAsyncU];
        bool ok[kAsyncU];
#pragma unroll
        for (int u = 0; u < kAsyncU; u++) {
            const uint32_t k = b0 + (uint32_t)(u * 32 + lane);
            int lo = 0;  // lanes whose inclusive prefix is <= k: the owner of item k
#pragma unroll
            for (int step = 16; step; step >>= 1) {
                const uint32_t pm = __shfl_sync(FULL, incl, lo + step - 1);
                if (pm <= k) lo += step;
            }
            const int32_t be = __shfl_sync(FULL, base_e, lo & 31);
            const float ds = __shfl_sync(FULL, du, lo & 31);
            const bool own_hub = (hubs >> (lo & 31)) & 1u;
            ok[u] = k < total;
            const int32_t e = be + (int32_t)k;
            if (ok[u] && own_hub) {  // a chunk of a claimed hub becomes dirty
                const int32_t c = e - V;
                const int32_t id = V + (c & 31) * a.nc32 + (c >> 5);
                const uint32_t bit = 1u << ((id + order) & 31);
                if (!(atomicOr(&dirty[id >> 5], bit) & bit)) newly++;
                ok[u] = false;
            }
            x[u] = ok[u] ? __ldg(&a.col[e]) : 0;
            nd[u] = ok[u] ? ds + (kUnit ? 1.f : __ldg(&a.wt[e])) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < kAsyncU; u++) dx[u] = ok[u] ? ld_dist(a, x[u]) : 0.f;
        bool keep[kAsyncU];
#if MB_ASYNC_LOCAL == 2
        // a vertex that dropped below T is kept by this warp WITHOUT setting
        // its dirty bit (no publish, no claim back: two L2 round trips less
        // per hop of a light-edge chain); it counts as set in the work
        // counters until this warp relaxes it.  The rest are published.
        bool imp[kAsyncU];
#pragma unroll
        for (int u = 0; u < kAsyncU; u++) {
            imp[u] = false;
            if (ok[u] && nd[u] < dx[u]) {
                const unsigned old = atomicMin((unsigned *)&a.dist[x[u]], __float_as_uint(nd[u]));
                imp[u] = nd[u] < __uint_as_float(old);
            }
        }
#pragma unroll
        for (int u = 0; u < kAsyncU; u++) {
            const bool cand = imp[u] && nd[u] < T;
            const uint32_t km = __ballot_sync(FULL, cand);
            const uint32_t pos = *nn + __popc(km & lanemask_lt());
            keep[u] = cand && pos < kAsyncNext;
            if (keep[u]) {
                nxt[pos] = x[u];
                newly++;
            }
            *nn = min(kAsyncNext, *nn + (uint32_t)__popc(km));
            if (imp[u] && !keep[u]) {
                const uint32_t bit = 1u << ((x[u] + order) & 31);
                if (!(atomicOr(&dirty[x[u] >> 5], bit) & bit)) newly++;
            }
        }
#else
#pragma unroll
        for (int u = 0; u < kAsyncU; u++) {
            keep[u] = false;
            if (ok[u] && nd[u] < dx[u]) {
                const unsigned old = atomicMin((unsigned *)&a.dist[x[u]], __float_as_uint(nd[u]));
                if (nd[u] < __uint_as_float(old)) {
                    const uint32_t bit = 1u << ((x[u] + order) & 31);
                    if (!(atomicOr(&dirty[x[u] >> 5], bit) & bit)) {
                        newly++;
                        keep[u] = MB_ASYNC_LOCAL && nd[u] < T;
                    }
                }
            }
        }
#endif
        if (MB_ASYNC_LOCAL == 1) {
#pragma unroll
            for (int u = 0; u < kAsyncU; u++) {
                const uint32_t km = __ballot_sync(FULL, keep[u]);
                const uint32_t pos = *nn + __popc(km & lanemask_lt());
                if (keep[u] && pos < kAsyncNext) nxt[pos] = x[u];
                *nn = min(kAsyncNext, *nn + (uint32_t)__popc(km));
            }
        }
    }
    newly = warp_sum(newly);
    // performed after every bit set above (its operand depends on them)
    if (lane == 0 && (total | claimed))
        atomicAdd(&S->d[slot].v, (unsigned long long)(total - newly) + (unsigned long long)__popc(claimed));
    return total - warp_sum(hub ? deg : 0u);
}

// Lane 0 of a warp whose pass found nothing below the threshold, once per
// phase: count the warp idle; the CTA's last warp counts the CTA, and the
// grid's last CTA opens the next phase.
__device__ __forceinline__ void async_idle(Ctrl *c, AsyncState *S, uint32_t *s_idle, uint32_t ph,
                                           float T, float delta, float above, int cap) {
    uint32_t dep = 0;
    if (above < __uint_as_float(kInfBits))
        dep = atomicMin((unsigned *)&S->mn[ph & 1].v, __float_as_uint(above));
    // distances are non-negative: dep >> 31 is zero
    const uint32_t k = atomicAdd(&s_idle[ph & 1], 1u + (dep >> 31)) + 1u;
    if (k != (uint32_t)kAsyncWarps) return;
    // this CTA's warps all reported phase ph; none reports ph + 1 before the
    // phase opens, which needs this CTA's count below
    const uint32_t r = atomicExch(&s_idle[(ph + 1) & 1], 0u);
    __threadfence();
    const uint32_t g = atomicAdd((unsigned *)&S->idle[ph & 1].v, 1u + (r >> 31)) + 1u;
    if (g != gridDim.x) return;
    // every CTA idle in phase ph: raise the threshold
    const uint32_t mb = atomicExch((unsigned *)&S->mn[ph & 1].v, kInfBits);
    const float m = __uint_as_float(mb);
    float tn = T + delta;
    if (m < __uint_as_float(kInfBits) && m + delta > tn) tn = m + delta;
    // where a sum rounds back (distances past 2^24, a small step), one float
    // step past the least distance seen above T, so that vertex is below tn
    if (!(tn > T)) tn = __uint_as_float(__float_as_uint(T) + 1u);
    if (m < __uint_as_float(kInfBits) && !(tn > m)) tn = __uint_as_float(mb + 1u);
    const uint32_t r2 = atomicExch((unsigned *)&S->idle[(ph + 1) & 1].v, 0u);
    const uint32_t nph = ph + 1u + (r2 >> 31) + (mb >> 31);  // both shifts zero
    atomicExch(&S->pt.v, ((unsigned long long)nph << 32) | __float_as_uint(tn));
    atomicAdd(&c->splits, 1);
    atomicAdd(&c->supersteps, 1);
    if ((int64_t)nph > (int64_t)cap) async_abort(c, S, ERR_STEP_CAP);
}

// kUnit: every weight 1 (BFS levels as hop distances; a.wt is not read).
template <bool kUnit>
__global__ void __launch_bounds__(kAsyncThreads) k_sssp_async(SsspArgs a, int cap) {
    const unsigned FULL = 0xffffffffu;
    Ctrl *c = a.f.ctrl;
    count_launch(c);
    AsyncState *S = a.as;
    uint32_t *dirty = a.adirty;
    __shared__ uint32_t s_idle[2];
    __shared__ int s_ok;
    __shared__ volatile int s_done;  // set by the CTA's checker warp: every warp leaves
    // claimed vertices waiting for a full batch of 32, and the vertices the
    // warp keeps for itself (local continuation), per warp
    __shared__ int32_t s_bv[kAsyncWarps][64];
    __shared__ int32_t s_nxt[kAsyncWarps][kAsyncNext];
    int32_t *bv = s_bv[threadIdx.x >> 5];
    int32_t *nxt = s_nxt[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = gridDim.x * kAsyncWarps;
    const uint32_t gw = blockIdx.x * kAsyncWarps + (threadIdx.x >> 5);
    const int slot = (int)(gw & (kAsyncSlots - 1));
    const long budget = c->p.wait_polls >= 0 ? (long)c->p.wait_polls : kAsyncSpins;
    const float delta = c->p.async_delta;
    const float inf = __uint_as_float(kInfBits);
    const int64_t W = a.WA;
    const int32_t V = a.f.V;
    if (threadIdx.x < 2) s_idle[threadIdx.x] = 0u;
    if (threadIdx.x == 0) s_done = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0)  // finish_superstep credits the frontier's edges
        atomicAdd((unsigned long long *)&c->work, 0ull - (unsigned long long)c->front_m);
    // 1. the queue frontier's vertices become dirty
    {
        const int cur = c->cur;
        const uint32_t n = (uint32_t)(c->q[cur] >> 32);
        const int32_t *qv = pick(a.f.qv, cur);
        uint32_t again = 0;
        float dmin = inf;
        for (uint32_t b0 = gw * 32u; b0 < n; b0 += nwarps * 32u) {
            const uint32_t i = b0 + (uint32_t)lane;
            const bool ok = i < n;
            const int32_t v = ok ? qv[i] : 0;
            const unsigned m = __ballot_sync(FULL, ok);
            unsigned long long pre = 0;
            if (lane == 0) pre = atomicAdd(&S->p[slot].v, (unsigned long long)__popc(m));
            const int32_t order = (int32_t)(__shfl_sync(FULL, pre, 0) >> 63);
            if (ok) {
                dmin = fminf(dmin, ld_dist(a, v));
                const uint32_t bit = 1u << ((v + order) & 31);
                if (atomicOr(&dirty[v >> 5], bit) & bit) again++;
            }
        }
        again = warp_sum(again);
        dmin = warp_min_f(dmin);
        if (lane == 0) {
            if (again) atomicAdd(&S->d[slot].v, (unsigned long long)again);
            if (dmin < inf) atomicMin((unsigned *)&S->t0.v, __float_as_uint(dmin));
            __threadfence();
        }
    }
    // 2. start barrier (bounded)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd((unsigned *)&S->bar.v, 1u);
        int ok = 0;
        for (long it = 0;; it++) {
            if (ld_acquire_gpu((const unsigned *)&S->bar.v) >= gridDim.x) {
                ok = 1;
                break;
            }
            if (it >= budget) break;
            __nanosleep(32);
        }
        if (!ok) async_abort(c, S, ERR_ASYNC);
        s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) return;
    const float t0 = __uint_as_float(ld_rlx32(&S->t0.v));
    const float T0 = delta > 0.f ? t0 + delta : inf;
    // 3. claim and relax until no work is left
    uint32_t reported = 0xffffffffu;
    long idle = 0, busy = 0;
    unsigned long long relaxed = 0;
    const bool checker = (threadIdx.x >> 5) == 0;
    for (;;) {
        if (s_done) break;
        // warp 0 of each CTA, after an idle pass, looks for the end of the
        // run (every fourth idle pass: the test reads 64 counter lines) or
        // an abort, and tells the CTA's other warps through shared memory
        if (checker && idle > 0) {
            bool fin = ld_rlx32(&S->abort_.v) != 0u;
            if (!fin && (idle & 3) == 1) fin = async_finished(S);
            if (fin) {
                if (lane == 0) s_done = 1;
                break;
            }
        }
        const unsigned long long pt = ld_rlx64(&S->pt.v);
        const uint32_t ph = (uint32_t)(pt >> 32);
        const float T = ph ? __uint_as_float((uint32_t)pt) : T0;
        bool found = false;
        float above = inf;
        uint32_t nb = 0;  // vertices in bv (warp-uniform)
        uint32_t nn = 0;  // vertices in nxt (warp-uniform)
        // relax full batches of bv (all of it when `all`), taking the kept
        // vertices of nxt into bv (claimed back from the bitmap) as they come
        auto drain = [&](bool all) {
            for (;;) {
                if (nn > 0 && nb < 32) {
                    const uint32_t take = min(nn, 32u);
                    const int32_t x = lane < (int)take ? nxt[lane] : -1;
                    const int32_t rest = lane + (int)take < (int)nn ? nxt[lane + take] : -1;
                    __syncwarp();
                    if (lane + take < nn) nxt[lane] = rest;
                    nn -= take;
                    bool got = false;
                    if (x >= 0) {
#if MB_ASYNC_LOCAL == 2
                        got = true;  // never published: no claim needed
#else
                        const uint32_t bit = 1u << (x & 31);
                        got = (atom_and_acquire(&dirty[x >> 5], ~bit) & bit) != 0u;
#endif
                    }
                    const uint32_t gm = __ballot_sync(FULL, got);
                    if (got) bv[nb + __popc(gm & lanemask_lt())] = x;
                    nb += __popc(gm);
                    __syncwarp();
                    continue;
                }
                if (nb >= 32 || (all && nb > 0)) {
                    relaxed += async_relax<kUnit>(a, S, slot, lane < (int)nb ? bv[lane] : -1, T, nxt, &nn);
                    const uint32_t done = min(nb, 32u);
                    const uint32_t rest = nb - done;
                    const int32_t t = lane < (int)rest ? bv[32 + lane] : -1;
                    __syncwarp();
                    if (lane < (int)rest) bv[lane] = t;
                    nb = rest;
                    __syncwarp();
                    continue;
                }
                break;
            }
        };
        for (int64_t b0 = gw; b0 < W; b0 += (int64_t)nwarps * 32) {
            const int64_t wl = b0 + (int64_t)lane * nwarps;
            const uint32_t xl = wl < W ? __ldcg(&dirty[wl]) : 0u;
            uint32_t nz = __ballot_sync(FULL, xl != 0u);
            while (nz) {
                const int j = __ffs(nz) - 1;
                nz &= nz - 1;
                const int64_t w = b0 + (int64_t)j * nwarps;
                const uint32_t x = __shfl_sync(FULL, xl, j);
                const bool has = (x >> lane) & 1u;
                const int32_t id = (int32_t)(w * 32 + lane);
                const float d = !has ? inf : ld_dist(a, id < V ? id : __ldg(&a.chunk_src[id - V]));
                const bool below = has && d < T;
                if (has && !below) above = fminf(above, d);
                const uint32_t mask = __ballot_sync(FULL, below);
                if (!mask) continue;
                uint32_t old = 0;
                if (lane == 0) old = atom_and_acquire(&dirty[w], ~mask);
                const uint32_t claimed = __shfl_sync(FULL, old, 0) & mask;
                if (!claimed) continue;
                found = true;
                if ((claimed >> lane) & 1u) bv[nb + __popc(claimed & lanemask_lt())] = id;
                nb += __popc(claimed);
                __syncwarp();
                drain(false);
            }
        }
        drain(true);
        if (found) {
            idle = 0;
            if (++busy > (long)cap) {  // more claiming passes than supersteps allowed
                if (lane == 0) {
                    async_abort(c, S, ERR_STEP_CAP);
                    s_done = 1;
                }
                break;
            }
            continue;
        }
        if (reported != ph) {
            reported = ph;
            above = warp_min_f(above);
            if (lane == 0) async_idle(c, S, s_idle, ph, T, delta, above, cap);
            __syncwarp();
        }
        if (++idle > budget) {
            if (lane == 0) {
                async_abort(c, S, ERR_ASYNC);
                s_done = 1;
            }
            break;
        }
        __nanosleep(128u << (idle < MB_ASYNC_SLEEP_MAX ? idle : MB_ASYNC_SLEEP_MAX));
    }
    if (lane == 0 && relaxed) atomicAdd((unsigned long long *)&c->work, relaxed);
}

// Hub chunk tables of the asynchronous kernel (once per graph).
__global__ void k_chunk_count(const int32_t *row, int32_t V, uint32_t *cnt) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t deg = row[v + 1] - row[v];
        cnt[v] = deg > kAsyncChunk ? (uint32_t)((deg + kAsyncChunk - 1) / kAsyncChunk) : 0u;
    }
}
__global__ void k_chunk_fill(const int32_t *row, int32_t V, const int32_t *cbase, int32_t nc32,
                             int32_t *csrc, int32_t *crs) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t rs = row[v], deg = row[v + 1] - rs;
        if (deg <= kAsyncChunk) continue;
        const int32_t n = (deg + kAsyncChunk - 1) / kAsyncChunk, c0 = cbase[v];
        for (int32_t j = 0; j < n; j++) {
            const int32_t c = c0 + j, q = (c & 31) * nc32 + (c >> 5);
            csrc[q] = (int32_t)v;
            crs[q] = rs + j * kAsyncChunk;
        }
    }
}
