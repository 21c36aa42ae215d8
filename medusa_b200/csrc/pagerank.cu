// pagerank.cu -- the PageRank app's BSP superstep on sm_100a.
//
// Reference (MPG/UserOperators.h:16-43,119-144,175-270; combiner with
// CUDPP_ADD; CPU form MPG/CPUFunctorHoster.cpp:17-31,60-93,143-163):
//   send    msg = rank[u] / outdeg[u] (float) on every out-edge of u
//   combine sum of the messages of each destination
//   update  rank[v] = 0.15 + 0.85 * sum, with the reference's rounding:
//           sum *= 0.85 is a double multiply rounded to float, and
//           0.15 + sum a double add rounded to float.
// No dangling-rank redistribution; a vertex with no in-edges gets 0.15.
//
// The sum runs in the fixed order of pr_order.cuh, the same for every
// schedule, so schedules never change a bit of the result.  Work mapping:
//   light vertices (in-degree <= kPrLight): their in-edge sources are copied
//     once per graph into a compacted list; one warp per 32 x VPL (1, 2 or
//     4) consecutive light vertices streams their in-edges through a
//     shared-memory window (coalesced) and each lane folds its own vertices
//     (k_pr_light; the message-reading schedule uses k_pr_pull over the
//     full reverse CSR);
//   heavier vertices: their kPrBlock-edge blocks form a work list built once
//     per graph, one 16-byte item per block (edge range, vertex, slot); one
//     warp per long item, or 1, 2 or 4 short items per warp
//     (k_heavy_blocks).  A vertex with a single block is
//     finished there (update and next contribution); a hub's blocks write
//     block sums that k_hub_finalize folds in order -- so hubs and the long
//     tail of R-MAT's hundreds-to-thousands in-degrees spread over every SM
//     instead of serialising in one lane.
// Schedules: 0 fused pull (gather rank/outdeg, fold, update, write the next
// contribution); 6 the reference's split: send into the E-slot message
// array at msgDstID, then the same combine+update reading the messages.
#include <algorithm>
#include <vector>
#include "pagerank.cuh"
#include "pr_order.cuh"

namespace mb {
namespace {

constexpr int kWin = 512;                // edges staged per warp per window
constexpr int kPrWarps = 8;              // warps per CTA
constexpr int kPrThreads = kPrWarps * 32;

struct PrArgs {
    int32_t V;
    int64_t E;
    const int32_t *rrow, *rcol, *outdeg, *row, *mslot;  // rcol/mslot: of the order in use
    const float *contrib_in;   // rank[u]/outdeg[u] of the previous superstep
    float *contrib_out;
    float *rank_out;
    float *msg;                // E-slot message array (schedule 6)
    const int4 *items;           // heavy blocks: {j0, j1, vertex, hub slot or -1}
    int32_t nitems;
    const int32_t *hub_v;        // vertices with more than one block
    const int32_t *hub_first;    // first slot of each hub (nhub+1 entries)
    int32_t nhub;
    float *blk_sum;              // per-slot block sums of the hubs
    int32_t nlong;               // items [0, nlong) are longer than kPrShortItem
    const int32_t *light_v;      // light vertices, id order
    const int32_t *light_row;    // their in-edge offsets into light_col (nlight+1)
    const int32_t *light_col;    // their in-edge sources, reverse-CSR order
    int32_t nlight;
};

__device__ __forceinline__ void pr_write(const PrArgs &a, int32_t v, float sum, int32_t d) {
    const float r = pr_update(sum);
    a.rank_out[v] = r;
    a.contrib_out[v] = d > 0 ? r / (float)d : 0.0f;  // MPG/CPUFunctorHoster.cpp:80-82
}

__device__ __forceinline__ void pr_write(const PrArgs &a, int32_t v, float sum) {
    pr_write(a, v, sum, a.outdeg[v]);
}

// Streamed index arrays (read once per superstep) bypass L1, which is left
// to the contribution gathers: a hot source's contribution then stays in L1
// for the next warps that gather it (4% at 2^28 edges; an evict_last hint on
// the gathers measured 5% slower).
__device__ __forceinline__ int32_t ld_stream(const int32_t *p) {
    int32_t v;
    asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ float ld_gather(const float *p) { return __ldg(p); }

template <bool kFromMsg>
__device__ __forceinline__ float edge_val(const PrArgs &a, int64_t j) {
    if (kFromMsg) return a.msg[j];
    return ld_gather(&a.contrib_in[ld_stream(&a.rcol[j])]);
}

// Heavy-vertex blocks (<= kPrBlock in-edges each), summed exactly as
// pr_warp_block_sum does: lane l folds edges l, l+32, ... from 0, then the
// xor butterfly.  The list is sorted longest first.  Its head (items longer
// than kPrShortItem) takes one item per warp with kLongU loads of each lane
// in flight; the rest take kShortPair items per warp at once (kShortU loads
// of each item in flight), so short items do not leave a warp waiting on a
// handful of loads.  Neither grouping changes a bit.  A single-block vertex
// is finished here; a hub block writes its block sum.
#ifndef MB_PR_LONG_UNROLL
#define MB_PR_LONG_UNROLL 16
#endif
constexpr int kLongU = MB_PR_LONG_UNROLL;
constexpr int kShortU = 4;
constexpr int kPrShortItem = 32 * kShortU * 4;  // 512 edges
constexpr int kShortPairDefault = 2;  // measured best at 2^20-2^28 edges

__host__ __device__ __forceinline__ int64_t heavy_units(int32_t nitems, int32_t nlong, int pair) {
    return (int64_t)nlong + ((int64_t)nitems - nlong + pair - 1) / pair;
}

__device__ __forceinline__ void heavy_finish(const PrArgs &a, const int4 &it, float acc, int32_t d) {
    if (it.w == -2) return;  // past the list
    if (it.w < 0) pr_write(a, it.z, 0.f + acc, d);  // one block sum folded from 0
    else a.blk_sum[it.w] = acc;
}

template <bool kFromMsg, int kShortPair>
__global__ void __launch_bounds__(256) k_heavy_blocks(PrArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t units = heavy_units(a.nitems, a.nlong, kShortPair);
    for (int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; u < units; u += warps) {
        if (u < a.nlong) {
            const int4 it = __ldg(&a.items[u]);
            const int32_t d = (lane == 0 && it.w < 0) ? __ldg(&a.outdeg[it.z]) : 0;
            const int32_t len = it.y - it.x;
            float acc = 0.f;
            for (int32_t k0 = 0; k0 < len; k0 += 32 * kLongU) {
                float val[kLongU];
#pragma unroll
                for (int q = 0; q < kLongU; q++) {
                    const int32_t k = k0 + lane + 32 * q;
                    val[q] = k < len ? edge_val<kFromMsg>(a, (int64_t)it.x + k) : 0.f;
                }
#pragma unroll
                for (int q = 0; q < kLongU; q++)
                    if (k0 + lane + 32 * q < len) acc += val[q];
            }
#pragma unroll
            for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
            if (lane == 0) heavy_finish(a, it, acc, d);
            continue;
        }
        const int64_t b0 = a.nlong + (u - a.nlong) * kShortPair;
        int4 it[kShortPair];
        int32_t len[kShortPair], d[kShortPair], lmax = 0;
        float acc[kShortPair];
#pragma unroll
        for (int p = 0; p < kShortPair; p++) {
            it[p] = b0 + p < a.nitems ? __ldg(&a.items[b0 + p]) : make_int4(0, 0, 0, -2);
            len[p] = it[p].y - it[p].x;
            lmax = max(lmax, len[p]);
            acc[p] = 0.f;
        }
#pragma unroll
        for (int p = 0; p < kShortPair; p++)
            d[p] = (lane == 0 && it[p].w == -1) ? __ldg(&a.outdeg[it[p].z]) : 0;
        for (int32_t k0 = 0; k0 < lmax; k0 += 32 * kShortU) {
            float val[kShortPair][kShortU];
#pragma unroll
            for (int p = 0; p < kShortPair; p++)
#pragma unroll
                for (int q = 0; q < kShortU; q++) {
                    const int32_t k = k0 + lane + 32 * q;
                    val[p][q] = k < len[p] ? edge_val<kFromMsg>(a, (int64_t)it[p].x + k) : 0.f;
                }
#pragma unroll
            for (int p = 0; p < kShortPair; p++)
#pragma unroll
                for (int q = 0; q < kShortU; q++)
                    if (k0 + lane + 32 * q < len[p]) acc[p] += val[p][q];
        }
#pragma unroll
        for (int p = 0; p < kShortPair; p++) {
#pragma unroll
            for (int off = 16; off; off >>= 1) acc[p] += __shfl_xor_sync(0xffffffffu, acc[p], off);
        }
        if (lane == 0) {
#pragma unroll
            for (int p = 0; p < kShortPair; p++) heavy_finish(a, it[p], acc[p], d[p]);
        }
    }
}

// Hubs (more than one block): fold the block sums in order, then update.
__global__ void k_hub_finalize(PrArgs a) {
    for (int32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < a.nhub; h += gridDim.x * blockDim.x) {
        float sum = 0.f;
        for (int32_t k = a.hub_first[h]; k < a.hub_first[h + 1]; k++) sum += a.blk_sum[k];
        pr_write(a, a.hub_v[h], sum);
    }
}

// Combine+update over the full reverse CSR (the message-reading schedule and
// the reference's MEG order): one warp per 32 consecutive vertices.  The warp
// streams the group's in-edges (contiguous in reverse-CSR order) through a
// shared-memory window, coalesced; each lane then folds its own vertex's
// part of the window in order.  kAllLight (the reference's MEG order): every
// vertex, hubs included, is folded sequentially by its lane.
template <bool kFromMsg, bool kAllLight = false>
__global__ void __launch_bounds__(kPrThreads) k_pr_pull(PrArgs a) {
    __shared__ float win[kPrWarps][kWin];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float *wv = win[wid];
    const int64_t ngroups = ((int64_t)a.V + 31) / 32;
    const int64_t warps = (int64_t)gridDim.x * kPrWarps;
    for (int64_t grp = (int64_t)blockIdx.x * kPrWarps + wid; grp < ngroups; grp += warps) {
        const int32_t v = (int32_t)(grp * 32 + lane);
        const bool valid = v < a.V;
        const int32_t vb = (int32_t)(grp * 32);
        const int32_t ve = (int32_t)min(grp * 32 + 32, (int64_t)a.V);
        int64_t b = 0, e = 0;
        if (valid) {
            b = a.rrow[v];
            e = a.rrow[v + 1];
        }
        const bool heavy = !kAllLight && valid && (e - b) > kPrLight;
        const int64_t g0 = a.rrow[vb], g1 = a.rrow[ve];
        float sum = 0.f;
        // heavy vertices are finished by k_heavy_blocks / k_hub_finalize
        for (int64_t w0 = g0; w0 < g1; w0 += kWin) {
            const int64_t w1 = min(w0 + (int64_t)kWin, g1);
            // skip windows that lie entirely inside heavy ranges
            const bool mine = !heavy && b < w1 && e > w0;
            if (!__any_sync(0xffffffffu, mine)) continue;
            // every load of the window in flight at once
            float vals[kWin / 32];
#pragma unroll
            for (int r = 0; r < kWin / 32; r++) {
                const int64_t j = w0 + lane + 32 * r;
                vals[r] = j < w1 ? edge_val<kFromMsg>(a, j) : 0.f;
            }
#pragma unroll
            for (int r = 0; r < kWin / 32; r++) wv[lane + 32 * r] = vals[r];
            __syncwarp();
            if (mine) {
                const int64_t lo = max(b, w0), hi = min(e, w1);
                for (int64_t j = lo; j < hi; j++) sum += wv[j - w0];
            }
            __syncwarp();
        }
        if (valid && !heavy) pr_write(a, v, sum);
    }
}

// Fused combine+update of the light vertices (in-degree <= kPrLight) from
// the compacted light lists: one warp per group of 32 * kVPL consecutive
// light vertices (lane l owns the group's vertices l, l+32, ...).  The warp
// streams the group's in-edge sources (contiguous in light_col) through a
// shared-memory window of gathered contributions, every load of a window in
// flight at once, and each lane folds its vertices' parts of the window in
// order: the sequential fold of pr_order.cuh.
template <int kVPL>
__global__ void __launch_bounds__(kPrThreads) k_pr_light(PrArgs a) {
    __shared__ float win[kPrWarps][kWin];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float *wv = win[wid];
    constexpr int kG = 32 * kVPL;
    const int64_t ngroups = ((int64_t)a.nlight + kG - 1) / kG;
    const int64_t warps = (int64_t)gridDim.x * kPrWarps;
    for (int64_t grp = (int64_t)blockIdx.x * kPrWarps + wid; grp < ngroups; grp += warps) {
        const int32_t i0 = (int32_t)(grp * kG);
        const int32_t iend = (int32_t)min((int64_t)i0 + kG, (int64_t)a.nlight);
        int32_t v[kVPL], b[kVPL], e[kVPL], d[kVPL];
        float sum[kVPL];
#pragma unroll
        for (int i = 0; i < kVPL; i++) {
            const int32_t idx = i0 + 32 * i + lane;
            v[i] = -1;
            b[i] = e[i] = 0;
            sum[i] = 0.f;
            if (idx < iend) {
                v[i] = ld_stream(&a.light_v[idx]);
                b[i] = ld_stream(&a.light_row[idx]);
                e[i] = ld_stream(&a.light_row[idx + 1]);
            }
        }
#pragma unroll
        for (int i = 0; i < kVPL; i++) d[i] = v[i] >= 0 ? __ldg(&a.outdeg[v[i]]) : 0;
        const int32_t g0 = __ldg(&a.light_row[i0]), g1 = __ldg(&a.light_row[iend]);
        for (int32_t w0 = g0; w0 < g1; w0 += kWin) {
            const int32_t w1 = min(w0 + kWin, g1);
            int32_t src[kWin / 32];
#pragma unroll
            for (int r = 0; r < kWin / 32; r++) {
                const int32_t j = w0 + lane + 32 * r;
                src[r] = j < w1 ? ld_stream(&a.light_col[j]) : -1;
            }
            float vals[kWin / 32];
#pragma unroll
            for (int r = 0; r < kWin / 32; r++) vals[r] = src[r] >= 0 ? ld_gather(&a.contrib_in[src[r]]) : 0.f;
#pragma unroll
            for (int r = 0; r < kWin / 32; r++) wv[lane + 32 * r] = vals[r];
            __syncwarp();
#pragma unroll
            for (int i = 0; i < kVPL; i++) {
                const int32_t lo = max(b[i], w0), hi = min(e[i], w1);
                for (int32_t j = lo; j < hi; j++) sum[i] += wv[j - w0];
            }
            __syncwarp();
        }
#pragma unroll
        for (int i = 0; i < kVPL; i++)
            if (v[i] >= 0) pr_write(a, v[i], sum[i], d[i]);
    }
}

// ---- the reference's order (MB_PR_ORDER_REFERENCE), in parallel -------------
// Every vertex's sum is the reference's sequential float fold over its MEG
// slots, bit for bit (pr_order.cuh).  Three mappings by in-degree n:
//   n <= kPrLight: k_pr_light over light lists copied from the MEG order;
//   kPrLight < n <= hub_min: sliced ELL -- vertices sorted by in-degree, 32
//     per group; row j of a group holds slot j of each of its vertices, so a
//     warp reads a row with one coalesced load and lane l folds its own
//     vertex in order (k_pr_sell, on a second side stream beside the light
//     kernel);
//   n > hub_min: the contributions staged by every SM into one contiguous run
//     per vertex (k_pr_hub_stage), then one CTA per vertex runs the parallel
//     integer scan of pr_order.cuh over it (k_pr_hub_exact), on a side
//     stream beside the others.
#ifndef MB_SELL_U
#define MB_SELL_U 16
#endif
constexpr int kSellU = MB_SELL_U;               // rows of a group in flight
constexpr int kHubK = 16;                       // consecutive slots per thread
constexpr int kHubBig = 16384;                  // in-degree above which a hub gets the big CTA
constexpr int kHubMinDefault = 2048;

struct ExactArgs {
    const int32_t *rrow, *meg_src, *outdeg;
    const float *contrib_in;
    float *contrib_out, *rank_out;
    const int32_t *sell_v;       // 32 vertices per group (-1: padding), sorted by in-degree
    const int64_t *sell_base;    // first element of each group in sell_src
    const int32_t *sell_rows;    // rows of each group (its largest in-degree)
    const int32_t *sell_src;     // group g, row j, lane l at sell_base[g] + 32 j + l (-1: padding)
    int32_t ngroups;
    const int32_t *hub_v;        // hubs, largest in-degree first
    int32_t nhub;
    float *x_stage;              // every hub's contributions, in MEG slot order
    const int64_t *stage_off;    // where hub h's run starts (16-byte aligned)
    const int4 *stage_items;     // staging work: {stage offset, meg_src offset, length, 0}
    int32_t nstage_items;
};

__device__ __forceinline__ void x_write(const ExactArgs &a, int32_t v, float sum, int32_t d) {
    const float r = pr_update(sum);
    a.rank_out[v] = r;
    a.contrib_out[v] = d > 0 ? r / (float)d : 0.0f;
}

// Sliced ELL: one warp per group, kSellU rows (coalesced index loads, then
// the gathers) in flight; each lane folds its own vertex's slots in order.
// Padding slots (-1) read 0, and s + 0 = s, so they change no bit.
__global__ void __launch_bounds__(256) k_pr_sell(ExactArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < a.ngroups; g += warps) {
        const int32_t v = __ldg(&a.sell_v[g * 32 + lane]);
        const int32_t rows = __ldg(&a.sell_rows[g]);
        const int32_t d = v >= 0 ? __ldg(&a.outdeg[v]) : 0;
        const int32_t *src = a.sell_src + __ldg(&a.sell_base[g]) + lane;
        float sum = 0.f;
        // the next rows' indices load while this block's gathers are in flight
        int32_t nxt[kSellU];
#pragma unroll
        for (int u = 0; u < kSellU; u++) nxt[u] = u < rows ? ld_stream(src + (int64_t)u * 32) : -1;
        for (int32_t j0 = 0; j0 < rows; j0 += kSellU) {
            int32_t idx[kSellU];
#pragma unroll
            for (int u = 0; u < kSellU; u++) idx[u] = nxt[u];
#pragma unroll
            for (int u = 0; u < kSellU; u++) {
                const int32_t j = j0 + kSellU + u;
                nxt[u] = j < rows ? ld_stream(src + (int64_t)j * 32) : -1;
            }
            float x[kSellU];
#pragma unroll
            for (int u = 0; u < kSellU; u++) x[u] = idx[u] >= 0 ? ld_gather(&a.contrib_in[idx[u]]) : 0.f;
#pragma unroll
            for (int u = 0; u < kSellU; u++) sum += x[u];
        }
        if (v >= 0) x_write(a, v, sum, d);
    }
}

// Staging: every hub's contributions gathered, in MEG slot order, into one
// contiguous run per hub (x_stage), by all SMs at once: one warp per item of
// at most kStageItem slots, kStageU loads of each lane in flight.  The
// scans below then read coalesced data instead of each hub's CTA gathering
// at one SM's rate.
#ifndef MB_STAGE_ITEM
#define MB_STAGE_ITEM 1024
#endif
// The sliced ELL runs on its own stream beside the light kernel and the hub
// scans, on half its resident grid.  Measured per 20 supersteps against the
// three in line on one stream: C5 27.7 against 28.0 ms, the C5 generator
// at 2^21 / 2^25 3.77 against 4.60, R-MAT 2^20 / 2^24 1.00 against 1.23
// (forked before the staging kernel instead, C5 lost 7%: the staging that
// the big hubs' scans wait for ran slower).
constexpr int kSellGridDiv = 2;  // C5: 24.0 ms per 20 supersteps, against 25.1 at 1 and 28.0 at 3
constexpr int kStageItem = MB_STAGE_ITEM;
constexpr int kStageU = 8;
__global__ void __launch_bounds__(256) k_pr_hub_stage(ExactArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t it = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < a.nstage_items; it += warps) {
        const int4 item = __ldg(&a.stage_items[it]);
        float *dst = a.x_stage + (uint32_t)item.x;
        const int32_t *src = a.meg_src + (uint32_t)item.y;
        for (int32_t k0 = 0; k0 < item.z; k0 += 32 * kStageU) {
            float x[kStageU];
#pragma unroll
            for (int u = 0; u < kStageU; u++) {
                const int32_t k = k0 + 32 * u + lane;
                x[u] = k < item.z ? ld_gather(&a.contrib_in[ld_stream(src + k)]) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kStageU; u++) {
                const int32_t k = k0 + 32 * u + lane;
                if (k < item.z) dst[k] = x[u];
            }
        }
    }
}

// Scan thread t's kHubK consecutive staged values of the chunk at `pos`
// (0 past the vertex's end).  run + pos is 16-byte aligned.
__device__ __forceinline__ void hub_load(const float *run, int32_t n, int32_t pos, int t, float (&x)[kHubK]) {
    const int32_t j0 = pos + t * kHubK;
    if (j0 + kHubK <= n) {
        const float4 *p4 = reinterpret_cast<const float4 *>(run + j0);
#pragma unroll
        for (int r = 0; r < kHubK / 4; r++) {
            const float4 t4 = __ldcs(p4 + r);
            x[4 * r] = t4.x;
            x[4 * r + 1] = t4.y;
            x[4 * r + 2] = t4.z;
            x[4 * r + 3] = t4.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kHubK; k++) x[k] = j0 + k < n ? __ldcs(run + j0 + k) : 0.f;
    }
}

// Hubs [h0, h1) of the list: one CTA of kT threads per vertex, over its
// staged run.  The first kHead values are folded by thread 0 (a multiple of
// 4, so the chunks that follow start 16-byte aligned); then chunks of
// kT * kHubK values, thread t owning kHubK consecutive ones, go through the
// integer scan of pr_order.cuh.  Each chunk's loads are issued one chunk
// ahead of its scan.
template <int kT, int kHead>
__global__ void __launch_bounds__(kT) k_pr_hub_exact(ExactArgs a, int32_t h0, int32_t h1) {
    static_assert(kHead % 4 == 0, "chunks start 16-byte aligned");
    constexpr int kW = kT / 32;
    constexpr int kChunk = kT * kHubK;
    __shared__ __align__(16) float head[kHead];
    __shared__ uint32_t wtot[kW];
    __shared__ int32_t wbad[kW];
    __shared__ float s_sh;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int32_t h = h0 + blockIdx.x; h < h1; h += gridDim.x) {
        const int32_t v = __ldg(&a.hub_v[h]);
        const int32_t n = __ldg(&a.rrow[v + 1]) - __ldg(&a.rrow[v]);
        const float *run = a.x_stage + __ldg(&a.stage_off[h]);
        const int32_t H = min(n, kHead);
        for (int i = tid; i < H; i += kT) head[i] = __ldcs(run + i);
        float x[kHubK], xn[kHubK];
        hub_load(run, n, H, tid, xn);  // the first chunk's loads go out before the head is folded
        __syncthreads();
        if (tid == 0) {  // the adds chain; the shared loads run ahead, 4 at a time
            float s0 = 0.f;
            const float4 *h4 = reinterpret_cast<const float4 *>(head);
            int i = 0;
#pragma unroll 8
            for (; i + 4 <= H; i += 4) {
                const float4 t = h4[i >> 2];
                s0 += t.x;
                s0 += t.y;
                s0 += t.z;
                s0 += t.w;
            }
            for (; i < H; i++) s0 += head[i];
            s_sh = s0;
        }
        __syncthreads();
        float s = s_sh;
        for (int32_t pos = H; pos < n; pos += kChunk) {
#pragma unroll
            for (int k = 0; k < kHubK; k++) x[k] = xn[k];
            if (pos + kChunk < n) hub_load(run, n, pos + kChunk, tid, xn);
            int start = 0;  // threads before it have folded their slots
            for (;;) {
                const uint32_t bits = __float_as_uint(s);
                const uint32_t ks = bits >> 23, base = (bits & 0x7fffffu) | 0x800000u;
                uint32_t L = 0;
                bool tie = false;
                if (tid >= start) {
#pragma unroll
                    for (int k = 0; k < kHubK; k++) L += pr_units(x[k], ks, tie);
                    L = min(L, 1u << 23);
                }
                // inclusive prefix over the CTA.  Up to the first bad thread it
                // stays below 2^24 + 2^23; past it a sum may wrap around 2^32,
                // which changes nothing: only the first bad thread is used
                uint32_t I = L;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, I, off);
                    if (lane >= off) I += y;
                }
                if (lane == 31) wtot[wid] = I;
                __syncthreads();
                uint32_t total = 0;
#pragma unroll
                for (int w = 0; w < kW; w++) {
                    const uint32_t t = wtot[w];
                    if (w < wid) I += t;
                    total += t;
                }
                const bool bad = tid >= start && (ks == 0 || ks == 255 || tie || base + I >= (1u << 24));
                const unsigned bm = __ballot_sync(0xffffffffu, bad);
                if (lane == 0) wbad[wid] = bm ? wid * 32 + __ffs(bm) - 1 : kT;
                __syncthreads();
                int c = kT;
#pragma unroll
                for (int w = 0; w < kW; w++) c = min(c, wbad[w]);
                if (c == kT) {  // the whole chunk stayed in the binade
                    s = pr_make(ks, base + total);
                    break;
                }
                if (tid == c) {  // the float path from the exact running sum
                    float s2 = c == start ? s : pr_make(ks, base + I - L);
#pragma unroll
                    for (int k = 0; k < kHubK; k++) s2 += x[k];
                    s_sh = s2;
                }
                __syncthreads();
                s = s_sh;
                start = c + 1;
                if (start >= kT) break;
            }
        }
        if (tid == 0) x_write(a, v, s, __ldg(&a.outdeg[v]));
        __syncthreads();  // head and s_sh are reused by the next hub
    }
}

// Hubs [h0, h1) of the list: one WARP per vertex over its staged run --
// the integer scan of pr_order.cuh with shuffles only (no CTA barrier), so
// a SM keeps dozens of hubs in flight.  Every lane first folds the first
// kWarpHead values itself (each value broadcast by a shuffle, the same adds
// in every lane); then chunks of 32 * kHubK values, lane l owning kHubK
// consecutive ones, loaded one chunk ahead of their scan.
constexpr int kWarpHead = 64;
__global__ void __launch_bounds__(256) k_pr_hub_warp(ExactArgs a, int32_t h0, int32_t h1) {
    constexpr int kChunk = 32 * kHubK;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t h = h0 + (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); h < h1; h += warps) {
        const int32_t v = __ldg(&a.hub_v[h]);
        const int32_t n = __ldg(&a.rrow[v + 1]) - __ldg(&a.rrow[v]);
        const float *run = a.x_stage + __ldg(&a.stage_off[h]);
        const int32_t H = min(n, kWarpHead);
        const float h_lo = lane < H ? __ldcs(run + lane) : 0.f;
        const float h_hi = lane + 32 < H ? __ldcs(run + lane + 32) : 0.f;
        float x[kHubK], xn[kHubK];
        hub_load(run, n, H, lane, xn);  // the first chunk's loads go out before the head is folded
        float s = 0.f;
        for (int i = 0; i < H; i++) s += __shfl_sync(0xffffffffu, i < 32 ? h_lo : h_hi, i & 31);
        for (int32_t pos = H; pos < n; pos += kChunk) {
#pragma unroll
            for (int k = 0; k < kHubK; k++) x[k] = xn[k];
            if (pos + kChunk < n) hub_load(run, n, pos + kChunk, lane, xn);
            int start = 0;  // lanes before it have folded their values
            for (;;) {
                const uint32_t bits = __float_as_uint(s);
                const uint32_t ks = bits >> 23, base = (bits & 0x7fffffu) | 0x800000u;
                uint32_t L = 0;
                bool tie = false;
                if (lane >= start) {
#pragma unroll
                    for (int k = 0; k < kHubK; k++) L += pr_units(x[k], ks, tie);
                    L = min(L, 1u << 23);
                }
                uint32_t I = L;  // inclusive prefix (< 2^28: 32 lanes of at most 2^23)
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, I, off);
                    if (lane >= off) I += y;
                }
                const uint32_t total = __shfl_sync(0xffffffffu, I, 31);
                const bool bad = lane >= start && (ks == 0 || ks == 255 || tie || base + I >= (1u << 24));
                const unsigned bm = __ballot_sync(0xffffffffu, bad);
                if (!bm) {  // the whole chunk stayed in the binade
                    s = pr_make(ks, base + total);
                    break;
                }
                const int c = __ffs(bm) - 1;
                float s2 = c == start ? s : pr_make(ks, base + I - L);
                if (lane == c) {  // the float path from the exact running sum
#pragma unroll
                    for (int k = 0; k < kHubK; k++) s2 += x[k];
                }
                s = __shfl_sync(0xffffffffu, s2, c);
                start = c + 1;
                if (start >= 32) break;
            }
        }
        if (lane == 0) x_write(a, v, s, __ldg(&a.outdeg[v]));
    }
}

// Group g of the sliced ELL: row j, lane l <- slot j of the group's vertex l.
__global__ void k_sell_fill(const int32_t *sell_v, const int64_t *sell_base, const int32_t *sell_rows,
                            int32_t ngroups, const int32_t *rrow, const int32_t *meg_src, int32_t *sell_src) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups; g += warps) {
        const int32_t v = sell_v[g * 32 + lane];
        const int32_t rows = sell_rows[g];
        const int64_t b = v >= 0 ? rrow[v] : 0;
        const int32_t n = v >= 0 ? rrow[v + 1] - (int32_t)b : 0;
        int32_t *dst = sell_src + sell_base[g] + lane;
        for (int32_t j = 0; j < rows; j++) dst[(int64_t)j * 32] = j < n ? meg_src[b + j] : -1;
    }
}

// Copy each light vertex's in-edge sources out of the reverse CSR.
__global__ void k_light_copy(const int32_t *light_v, const int32_t *light_row, int32_t nlight,
                             const int32_t *rrow, const int32_t *rcol, int32_t *light_col) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nlight;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = light_v[i], o = light_row[i];
        const int32_t b = rrow[v], n = rrow[v + 1] - b;
        for (int32_t k = 0; k < n; k++) light_col[o + k] = rcol[b + k];
    }
}

// Schedule 6, send (SendMsgAA, MPG/UserOperators.h:48-70): every vertex
// writes its contribution into the message slot of each out-edge.
__global__ void k_pr_send(PrArgs a) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < a.V;
         u += (int64_t)gridDim.x * blockDim.x) {
        const float m = a.contrib_in[u];
        for (int32_t e = a.row[u]; e < a.row[u + 1]; e++) a.msg[a.mslot[e]] = m;
    }
}

__global__ void k_pr_init(const int32_t *outdeg, int32_t V, float init, float *contrib) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < V;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = outdeg[u];
        contrib[u] = d > 0 ? init / (float)d : 0.0f;
    }
}

// The first superstep's contributions from a given rank vector.
__global__ void k_pr_init_vec(const int32_t *outdeg, int32_t V, const float *init, float *contrib) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < V;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = outdeg[u];
        contrib[u] = d > 0 ? init[u] / (float)d : 0.0f;
    }
}

__global__ void k_copy(float *dst, const float *src, int32_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

__global__ void k_fill(float *x, int32_t n, float v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] = v;
}

// MEG order, step 1: edge e (the k-th out-edge of u in reference order) has
// MEG position colstart[k] + rank[u]; order[pos] = e.
__global__ void k_meg_scatter(const int32_t *row, const int32_t *esrc, const int32_t *rank,
                              const int32_t *colstart, int64_t E, uint32_t *order) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = esrc[e];
        const int32_t k = (int32_t)(e - row[u]);
        order[(int64_t)colstart[k] + rank[u]] = (uint32_t)e;
    }
}

// step 2: (destination, edge) pairs in MEG position order, for the stable
// sort by destination
__global__ void k_meg_keys(const uint32_t *order, const int32_t *col, int64_t E, uint32_t *keys) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < E;
         i += (int64_t)gridDim.x * blockDim.x)
        keys[i] = (uint32_t)col[order[i]];
}

// step 3: slot p of the sorted sequence holds edge vals[p]
__global__ void k_meg_finish(const uint32_t *vals, const int32_t *esrc, int64_t E, int32_t *meg_src,
                             int32_t *meg_slot) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < E;
         p += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t e = vals[p];
        meg_src[p] = esrc[e];
        meg_slot[e] = (int32_t)p;
    }
}

}  // namespace

void build_meg_order(Context &ctx, const Graph &g, PrState &st) {
    if (st.meg_built) return;
    const int32_t V = g.V;
    const int64_t E = g.E;
    cudaStream_t s = ctx.stream;
    std::vector<int32_t> row((size_t)V + 1);
    copy_sync(ctx.stream, row.data(), g.row.p, sizeof(int32_t) * ((size_t)V + 1));
    // GraphIR::sortByDegree: std::sort of the vertices in id order by a
    // degree-descending comparator.  The permutation std::sort produces
    // depends only on the comparison results, so sorting (degree, id)
    // records with the same comparison reproduces the reference's.
    struct Node {
        int32_t deg, id;
    };
    std::vector<Node> nodes((size_t)V);
    for (int32_t v = 0; v < V; v++) nodes[v] = Node{row[v + 1] - row[v], v};
    std::sort(nodes.begin(), nodes.end(), [](const Node &l, const Node &r) { return l.deg > r.deg; });
    std::vector<int32_t> rank((size_t)V);
    for (int32_t i = 0; i < V; i++) rank[nodes[i].id] = i;
    // buildMEG: column k holds the k-th edge of every vertex with more than
    // k edges, in sorted order; colstart[k] = edges in columns before k
    const int32_t maxdeg = V ? nodes[0].deg : 0;
    std::vector<int64_t> cnt((size_t)maxdeg + 2, 0);
    for (int32_t v = 0; v < V; v++) cnt[row[v + 1] - row[v]]++;
    std::vector<int32_t> colstart((size_t)maxdeg + 1, 0);
    int64_t above = (int64_t)V - cnt[0], acc = 0;  // vertices with degree > k
    for (int32_t k = 0; k < maxdeg; k++) {
        colstart[k] = (int32_t)acc;
        acc += above;
        above -= cnt[k + 1];
    }
    colstart[maxdeg] = (int32_t)acc;
    DevBuf d_rank, d_col, order, keys;
    d_rank.reserve(sizeof(int32_t) * std::max<size_t>(V, 1));
    d_col.reserve(sizeof(int32_t) * colstart.size());
    const size_t eb = sizeof(uint32_t) * (size_t)std::max<int64_t>(E, 1);
    order.reserve(eb);
    keys.reserve(eb);
    st.meg_src.reserve(eb);
    st.meg_slot.reserve(eb);
    MB_CUDA(cudaMemcpyAsync(d_rank.p, rank.data(), sizeof(int32_t) * (size_t)V, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(d_col.p, colstart.data(), sizeof(int32_t) * colstart.size(), cudaMemcpyHostToDevice, s));
    if (E > 0) {
        const int grid = grid_for(E, 256, ctx.num_sms * 16);
        k_meg_scatter<<<grid, 256, 0, s>>>(g.row.as<int32_t>(), g.esrc.as<int32_t>(), d_rank.as<int32_t>(),
                                           d_col.as<int32_t>(), E, order.as<uint32_t>());
        k_meg_keys<<<grid, 256, 0, s>>>(order.as<uint32_t>(), g.col.as<int32_t>(), E, keys.as<uint32_t>());
        MB_CHECK_LAUNCH();
        int bits = 1;
        while (bits < 32 && ((int64_t)1 << bits) < (int64_t)V) bits++;
        radix_sort_pairs(ctx, keys.as<uint32_t>(), order.as<uint32_t>(), E, bits, s);
        k_meg_finish<<<grid, 256, 0, s>>>(order.as<uint32_t>(), g.esrc.as<int32_t>(), E,
                                          st.meg_src.as<int32_t>(), st.meg_slot.as<int32_t>());
        MB_CHECK_LAUNCH();
    }
    MB_CUDA(cudaStreamSynchronize(s));
    d_rank.release(); d_col.release(); order.release(); keys.release();
    st.meg_built = true;
}

void PrState::ensure(Context &ctx, const Graph &g) {
    if (built && V == g.V && E == g.E) return;
    release();
    V = g.V;
    E = g.E;
    rank.reserve(sizeof(float) * (size_t)V);
    contrib[0].reserve(sizeof(float) * (size_t)V);
    contrib[1].reserve(sizeof(float) * (size_t)V);
    msg.reserve(sizeof(float) * (size_t)std::max<int64_t>(E, 1));
    // heavy-vertex work list, built once per graph from the in-degree offsets:
    // one item per block; hubs (more than one block) get block-sum slots
    std::vector<int32_t> rrow(V + 1);
    copy_sync(ctx.stream, rrow.data(), g.rrow.p, sizeof(int32_t) * (V + 1));
    std::vector<int4> it;
    std::vector<int32_t> hv, hf;
    int32_t slots = 0;
    for (int32_t v = 0; v < V; v++) {
        const int64_t d = (int64_t)rrow[v + 1] - rrow[v];
        if (d <= kPrLight) continue;
        if (d <= kPrBlock) {
            it.push_back(make_int4(rrow[v], rrow[v + 1], v, -1));
            continue;
        }
        hv.push_back(v);
        hf.push_back(slots);
        for (int64_t j0 = rrow[v]; j0 < rrow[v + 1]; j0 += kPrBlock)
            it.push_back(make_int4((int32_t)j0, (int32_t)std::min<int64_t>(rrow[v + 1], j0 + kPrBlock),
                                   v, slots++));
    }
    hf.push_back(slots);
    // longest blocks first: the warps that take hub blocks start earliest
    // (the order of the items does not change any sum)
    std::stable_sort(it.begin(), it.end(),
                     [](const int4 &x, const int4 &y) { return (x.y - x.x) > (y.y - y.x); });
    nitems = (int32_t)it.size();
    nhub = (int32_t)hv.size();
    nlong = 0;
    while (nlong < nitems && it[nlong].y - it[nlong].x > kPrShortItem) nlong++;
    items.reserve(sizeof(int4) * std::max<size_t>(it.size(), 1));
    hub_v.reserve(sizeof(int32_t) * std::max<size_t>(hv.size(), 1));
    hub_first.reserve(sizeof(int32_t) * hf.size());
    blk_sum.reserve(sizeof(float) * std::max<int32_t>(slots, 1));
    copy_sync(ctx.stream, items.p, it.data(), sizeof(int4) * it.size());
    copy_sync(ctx.stream, hub_v.p, hv.data(), 4 * hv.size());
    copy_sync(ctx.stream, hub_first.p, hf.data(), 4 * hf.size());
    // light lists: the vertices with in-degree <= kPrLight and their in-edges
    std::vector<int32_t> lv, lr(1, 0);
    lv.reserve((size_t)V);
    lr.reserve((size_t)V + 1);
    for (int32_t v = 0; v < V; v++) {
        const int32_t d = rrow[v + 1] - rrow[v];
        if (d > kPrLight) continue;
        lv.push_back(v);
        lr.push_back(lr.back() + d);
    }
    nlight = (int32_t)lv.size();
    light_v.reserve(sizeof(int32_t) * std::max<size_t>(lv.size(), 1));
    light_row.reserve(sizeof(int32_t) * lr.size());
    light_col.reserve(sizeof(int32_t) * std::max<size_t>((size_t)lr.back(), 1));
    if (nlight) {
        copy_sync(ctx.stream, light_v.p, lv.data(), 4 * lv.size());
        copy_sync(ctx.stream, light_row.p, lr.data(), 4 * lr.size());
        k_light_copy<<<grid_for(nlight, 256, ctx.num_sms * 16), 256, 0, ctx.stream>>>(
            light_v.as<int32_t>(), light_row.as<int32_t>(), nlight, g.rrow.as<int32_t>(),
            g.rcol.as<int32_t>(), light_col.as<int32_t>());
        MB_CHECK_LAUNCH();
        MB_CUDA(cudaStreamSynchronize(ctx.stream));
    }
    built = true;
}

void PrState::ensure_exact(Context &ctx, const Graph &g, int32_t hub_min) {
    if (exact_built && x_hub_min == hub_min) return;
    build_meg_order(ctx, g, *this);
    release_exact();
    const int32_t V = g.V;
    cudaStream_t s = ctx.stream;
    std::vector<int32_t> rrow((size_t)V + 1);
    copy_sync(s, rrow.data(), g.rrow.p, sizeof(int32_t) * ((size_t)V + 1));
    // light vertices in id order, their sources copied out of the MEG order
    std::vector<int32_t> lv, lr(1, 0);
    // mid vertices by in-degree, largest first (ties in id order): a
    // counting sort over in-degrees kPrLight+1 .. hub_min
    std::vector<int64_t> cnt((size_t)hub_min + 2, 0);
    std::vector<int32_t> hubs;
    for (int32_t v = 0; v < V; v++) {
        const int32_t d = rrow[v + 1] - rrow[v];
        if (d <= kPrLight) {
            lv.push_back(v);
            lr.push_back(lr.back() + d);
        } else if (d <= hub_min) {
            cnt[d]++;
        } else {
            hubs.push_back(v);
        }
    }
    std::stable_sort(hubs.begin(), hubs.end(), [&](int32_t x, int32_t y) {
        return rrow[x + 1] - rrow[x] > rrow[y + 1] - rrow[y];
    });
    std::vector<int64_t> at((size_t)hub_min + 2, 0);
    int64_t nmid = 0;
    for (int32_t d = hub_min; d > kPrLight; d--) {
        at[d] = nmid;
        nmid += cnt[d];
    }
    std::vector<int32_t> mid((size_t)nmid);
    for (int32_t v = 0; v < V; v++) {
        const int32_t d = rrow[v + 1] - rrow[v];
        if (d > kPrLight && d <= hub_min) mid[at[d]++] = v;
    }
    ngroups = (int32_t)((nmid + 31) / 32);
    std::vector<int32_t> sv((size_t)ngroups * 32, -1), rows((size_t)ngroups);
    std::vector<int64_t> sbase((size_t)ngroups);
    int64_t total = 0;
    for (int32_t gi = 0; gi < ngroups; gi++) {
        for (int l = 0; l < 32 && (int64_t)gi * 32 + l < nmid; l++) sv[(size_t)gi * 32 + l] = mid[(size_t)gi * 32 + l];
        const int32_t v0 = sv[(size_t)gi * 32];
        rows[gi] = rrow[v0 + 1] - rrow[v0];
        sbase[gi] = total;
        total += (int64_t)rows[gi] * 32;
    }
    x_nlight = (int32_t)lv.size();
    x_light_v.reserve(sizeof(int32_t) * std::max<size_t>(lv.size(), 1));
    x_light_row.reserve(sizeof(int32_t) * lr.size());
    x_light_col.reserve(sizeof(int32_t) * std::max<size_t>((size_t)lr.back(), 1));
    sell_v.reserve(sizeof(int32_t) * std::max<size_t>(sv.size(), 1));
    sell_rows.reserve(sizeof(int32_t) * std::max<size_t>(rows.size(), 1));
    sell_base.reserve(sizeof(int64_t) * std::max<size_t>(sbase.size(), 1));
    sell_src.reserve(sizeof(int32_t) * (size_t)std::max<int64_t>(total, 1));
    x_nhub = (int32_t)hubs.size();
    x_hub_v.reserve(sizeof(int32_t) * std::max<size_t>(hubs.size(), 1));
    if (x_nlight) {
        copy_sync(s, x_light_v.p, lv.data(), 4 * lv.size());
        copy_sync(s, x_light_row.p, lr.data(), 4 * lr.size());
        k_light_copy<<<grid_for(x_nlight, 256, ctx.num_sms * 16), 256, 0, s>>>(
            x_light_v.as<int32_t>(), x_light_row.as<int32_t>(), x_nlight, g.rrow.as<int32_t>(),
            meg_src.as<int32_t>(), x_light_col.as<int32_t>());
        MB_CHECK_LAUNCH();
    }
    if (ngroups) {
        copy_sync(s, sell_v.p, sv.data(), 4 * sv.size());
        copy_sync(s, sell_rows.p, rows.data(), 4 * rows.size());
        copy_sync(s, sell_base.p, sbase.data(), 8 * sbase.size());
        k_sell_fill<<<grid_for((int64_t)ngroups * 32, 256, ctx.num_sms * 16), 256, 0, s>>>(
            sell_v.as<int32_t>(), sell_base.as<int64_t>(), sell_rows.as<int32_t>(), ngroups,
            g.rrow.as<int32_t>(), meg_src.as<int32_t>(), sell_src.as<int32_t>());
        MB_CHECK_LAUNCH();
    }
    if (x_nhub) copy_sync(s, x_hub_v.p, hubs.data(), 4 * hubs.size());
    x_nbig = 0;  // the hubs are sorted: the big ones come first
    while (x_nbig < x_nhub && rrow[hubs[x_nbig] + 1] - rrow[hubs[x_nbig]] > kHubBig) x_nbig++;
    // staging: hub h's run at a multiple of 4 floats, items of kStageItem slots
    std::vector<int64_t> soff((size_t)std::max<int32_t>(x_nhub, 1), 0);
    std::vector<int4> items;
    int64_t staged = 0;
    for (int32_t h = 0; h < x_nhub; h++) {
        const int32_t v = hubs[h];
        const int32_t n = rrow[v + 1] - rrow[v];
        soff[h] = staged;
        for (int32_t j0 = 0; j0 < n; j0 += kStageItem)
            items.push_back(make_int4((int32_t)(staged + j0), rrow[v] + j0, std::min(kStageItem, n - j0), 0));
        staged += ((int64_t)n + 3) & ~(int64_t)3;
    }
    if (staged > 0x7fffffffll) fail(MB_ERR_UNSUPPORTED, "PageRank: hub staging exceeds 2^31 slots");
    nstage_items = (int32_t)items.size();
    x_stage.reserve(sizeof(float) * (size_t)std::max<int64_t>(staged, 1));
    stage_off.reserve(sizeof(int64_t) * soff.size());
    stage_items.reserve(sizeof(int4) * std::max<size_t>(items.size(), 1));
    copy_sync(s, stage_off.p, soff.data(), 8 * soff.size());
    if (nstage_items) copy_sync(s, stage_items.p, items.data(), sizeof(int4) * items.size());
    MB_CUDA(cudaStreamSynchronize(s));
    ensure_streams();
    x_hub_min = hub_min;
    exact_built = true;
}

void run_pagerank(Context &ctx, Graph &g, PrState &st, int32_t iters, float init, int sched,
                  mb_stats *stats, const float *init_vec) {
    st.ensure(ctx, g);
    const bool ref_order = ctx.pr_order == MB_PR_ORDER_REFERENCE;
    const bool unfused = sched == MB_SCHED_PUSH_UNFUSED;
    const int32_t hub_min = ctx.tunable[MB_TUNE_PR_HUB_MIN] > 0
                                ? (int32_t)std::min<int64_t>(ctx.tunable[MB_TUNE_PR_HUB_MIN], 0x7fffffff)
                                : kHubMinDefault;
    if (ref_order) build_meg_order(ctx, g, st);
    if (ref_order && !unfused) st.ensure_exact(ctx, g, hub_min);
    st.ensure_streams();
    cudaStream_t s = ctx.stream;
    auto args = [&](int parity) {
        PrArgs a;
        a.V = g.V;
        a.E = g.E;
        a.rrow = g.rrow.as<int32_t>();
        a.rcol = ref_order ? st.meg_src.as<int32_t>() : g.rcol.as<int32_t>();
        a.outdeg = g.outdeg.as<int32_t>();
        a.row = g.row.as<int32_t>();
        a.mslot = ref_order ? st.meg_slot.as<int32_t>() : g.mslot.as<int32_t>();
        a.contrib_in = st.contrib[parity].as<float>();
        a.contrib_out = st.contrib[parity ^ 1].as<float>();
        a.rank_out = st.rank.as<float>();
        a.msg = st.msg.as<float>();
        a.items = st.items.as<int4>();
        a.nitems = st.nitems;
        a.hub_v = st.hub_v.as<int32_t>();
        a.hub_first = st.hub_first.as<int32_t>();
        a.nhub = st.nhub;
        a.blk_sum = st.blk_sum.as<float>();
        a.nlong = st.nlong;
        a.light_v = st.light_v.as<int32_t>();
        a.light_row = st.light_row.as<int32_t>();
        a.light_col = st.light_col.as<int32_t>();
        a.nlight = st.nlight;
        return a;
    };
    // grids of exactly the resident blocks (grid-stride loops: no tail wave)
    auto resident = [&](const void *k, int threads) {
        int per_sm = 0;
        MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, 0));
        return ctx.num_sms * std::max(per_sm, 1);
    };
    const int grid_pull = resident((const void *)k_pr_pull<false>, kPrThreads);
    // light vertices per lane: the tunable, else 2 (measured best from 2^22
    // to 2^28 edges) while every resident warp still gets four groups
    int vpl = (int)ctx.tunable[MB_TUNE_PR_LIGHT_VPL];
    if (vpl <= 0) {
        vpl = 2;
        const int64_t warps = (int64_t)resident((const void *)k_pr_light<1>, kPrThreads) * kPrWarps;
        const int64_t nl = ref_order && !unfused ? st.x_nlight : st.nlight;
        while (vpl > 1 && nl < (int64_t)32 * vpl * 4 * warps) vpl >>= 1;
    }
    const int pair = ctx.tunable[MB_TUNE_PR_SHORT_PAIR] > 0 ? (int)ctx.tunable[MB_TUNE_PR_SHORT_PAIR]
                                                             : kShortPairDefault;
    // each variant's grid is its own resident block count (registers differ)
    const void *heavy_fn[2][3] = {{(const void *)k_heavy_blocks<false, 1>, (const void *)k_heavy_blocks<false, 2>,
                                   (const void *)k_heavy_blocks<false, 4>},
                                  {(const void *)k_heavy_blocks<true, 1>, (const void *)k_heavy_blocks<true, 2>,
                                   (const void *)k_heavy_blocks<true, 4>}};
    const void *light_fn[3] = {(const void *)k_pr_light<1>, (const void *)k_pr_light<2>,
                               (const void *)k_pr_light<4>};
    const int pi = pair == 1 ? 0 : pair == 2 ? 1 : 2, vi = vpl == 1 ? 0 : vpl == 2 ? 1 : 2;
    const int64_t heavy_threads = heavy_units(st.nitems, st.nlong, pair) * 32;
    const int grid_heavy[2] = {grid_for(heavy_threads, 256, resident(heavy_fn[0][pi], 256)),
                               grid_for(heavy_threads, 256, resident(heavy_fn[1][pi], 256))};
    const int grid_light = resident(light_fn[vi], kPrThreads);
    auto heavy = [&](bool from_msg, cudaStream_t cs, const PrArgs &a) {
        PrArgs arg = a;
        void *params[] = {&arg};
        MB_CUDA(cudaLaunchKernel(heavy_fn[from_msg][pi], grid_heavy[from_msg], 256, params, 0, cs));
    };
    auto light = [&](cudaStream_t cs, const PrArgs &a) {
        PrArgs arg = a;
        void *params[] = {&arg};
        MB_CUDA(cudaLaunchKernel(light_fn[vi], grid_light, kPrThreads, params, 0, cs));
    };
    const int grid_vtx = ctx.num_sms * 8;
    const int grid_sell = resident((const void *)k_pr_sell, 256);
    const int hub_ctas = ctx.tunable[MB_TUNE_PR_HUB_CTAS] > 0 ? (int)ctx.tunable[MB_TUNE_PR_HUB_CTAS]
                                                               : std::max(ctx.num_sms / 4, 1);
    const int grid_hub_warp = std::max(resident((const void *)k_pr_hub_warp, 256) / 2, 1);
    const int grid_stage = resident((const void *)k_pr_hub_stage, 256);
    const int grid_hub_big = std::min(resident((const void *)k_pr_hub_exact<512, 512>, 512), hub_ctas);
    auto exact_args = [&](const PrArgs &a) {
        ExactArgs x;
        x.rrow = g.rrow.as<int32_t>();
        x.meg_src = st.meg_src.as<int32_t>();
        x.outdeg = g.outdeg.as<int32_t>();
        x.contrib_in = a.contrib_in;
        x.contrib_out = a.contrib_out;
        x.rank_out = a.rank_out;
        x.sell_v = st.sell_v.as<int32_t>();
        x.sell_base = st.sell_base.as<int64_t>();
        x.sell_rows = st.sell_rows.as<int32_t>();
        x.sell_src = st.sell_src.as<int32_t>();
        x.ngroups = st.ngroups;
        x.hub_v = st.x_hub_v.as<int32_t>();
        x.nhub = st.x_nhub;
        x.x_stage = st.x_stage.as<float>();
        x.stage_off = st.stage_off.as<int64_t>();
        x.stage_items = st.stage_items.as<int4>();
        x.nstage_items = st.nstage_items;
        return x;
    };
    auto emit = [&](cudaStream_t cs) {
        if (init_vec)
            k_pr_init_vec<<<grid_vtx, 256, 0, cs>>>(g.outdeg.as<int32_t>(), g.V, init_vec, st.contrib[0].as<float>());
        else
            k_pr_init<<<grid_vtx, 256, 0, cs>>>(g.outdeg.as<int32_t>(), g.V, init, st.contrib[0].as<float>());
        MB_CHECK_LAUNCH();
        for (int it = 0; it < iters; it++) {
            PrArgs a = args(it & 1);
            if (ref_order && unfused) {
                // the reference's send -> combine split over the message array,
                // each vertex folded serially in MEG order
                k_pr_send<<<grid_vtx, 256, 0, cs>>>(a);
                k_pr_pull<true, true><<<grid_pull, kPrThreads, 0, cs>>>(a);
                MB_CHECK_LAUNCH();
                continue;
            }
            if (ref_order) {
                ExactArgs x = exact_args(a);
                // the hubs' contributions staged by every SM, then their
                // scans on the side stream beside the rest
                const int32_t nbig = st.x_nbig, nsmall = st.x_nhub - st.x_nbig;
                if (st.x_nhub) {
                    k_pr_hub_stage<<<grid_stage, 256, 0, cs>>>(x);
                    MB_CHECK_LAUNCH();
                    MB_CUDA(cudaEventRecord(st.ev_fork, cs));
                    MB_CUDA(cudaStreamWaitEvent(st.side, st.ev_fork, 0));
                    // the scans beside the rest: the big hubs one CTA each on
                    // few CTAs, then the others one warp each
                    if (nbig)
                        k_pr_hub_exact<512, 512><<<std::min(nbig, grid_hub_big), 512, 0, st.side>>>(x, 0, nbig);
                    if (nsmall) {
                        // the warp scans beside the big hubs' CTAs when those
                        // take several rounds (more big hubs than CTAs);
                        // else after them (measured, 20 supersteps: C5, 301
                        // big hubs on 37 CTAs, 24.0 against 27.7 ms; the C5
                        // generator at 2^21, 22 big hubs, 4.10 against 3.79)
                        cudaStream_t hs = st.side;
                        if (nbig > grid_hub_big) {
                            MB_CUDA(cudaStreamWaitEvent(st.side3, st.ev_fork, 0));
                            hs = st.side3;
                        }
                        k_pr_hub_warp<<<grid_for((int64_t)nsmall * 32, 256, grid_hub_warp), 256, 0, hs>>>(
                            x, nbig, st.x_nhub);
                        if (hs == st.side3) {
                            MB_CUDA(cudaEventRecord(st.ev_join3, st.side3));
                            MB_CUDA(cudaStreamWaitEvent(st.side, st.ev_join3, 0));
                        }
                    }
                    MB_CHECK_LAUNCH();
                }
                // the sliced ELL on its own stream with half the GPU: its
                // longest groups (sequential folds) set its length, and the
                // light kernel fills the SMs its tail leaves idle
                if (st.ngroups) {
                    MB_CUDA(cudaEventRecord(st.ev_fork2, cs));
                    MB_CUDA(cudaStreamWaitEvent(st.side2, st.ev_fork2, 0));
                    k_pr_sell<<<std::max(grid_sell / kSellGridDiv, 1), 256, 0, st.side2>>>(x);
                    MB_CHECK_LAUNCH();
                }
                if (st.x_nlight) {
                    PrArgs la = a;
                    la.light_v = st.x_light_v.as<int32_t>();
                    la.light_row = st.x_light_row.as<int32_t>();
                    la.light_col = st.x_light_col.as<int32_t>();
                    la.nlight = st.x_nlight;
                    light(cs, la);
                }
                MB_CHECK_LAUNCH();
                if (st.x_nhub) {
                    MB_CUDA(cudaEventRecord(st.ev_join, st.side));
                    MB_CUDA(cudaStreamWaitEvent(cs, st.ev_join, 0));
                }
                if (st.ngroups) {
                    MB_CUDA(cudaEventRecord(st.ev_join2, st.side2));
                    MB_CUDA(cudaStreamWaitEvent(cs, st.ev_join2, 0));
                }
                continue;
            }
            if (unfused) {
                k_pr_send<<<grid_vtx, 256, 0, cs>>>(a);
                if (a.nitems) heavy(true, cs, a);
                k_pr_pull<true><<<grid_pull, kPrThreads, 0, cs>>>(a);
            } else {
                if (a.nitems) heavy(false, cs, a);
                if (a.nlight) light(cs, a);
            }
            if (a.nhub) k_hub_finalize<<<grid_for(a.nhub, 128, ctx.num_sms * 4), 128, 0, cs>>>(a);
            MB_CHECK_LAUNCH();
        }
        if (iters == 0) {  // no superstep: the ranks are the initial ranks
            if (init_vec) k_copy<<<grid_vtx, 256, 0, cs>>>(st.rank.as<float>(), init_vec, g.V);
            else k_fill<<<grid_vtx, 256, 0, cs>>>(st.rank.as<float>(), g.V, init);
            MB_CHECK_LAUNCH();
        }
    };
    cudaEvent_t e0, e1;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    try {
        if (ctx.use_graphs) {
            if (!st.exec || st.g_iters != iters || st.g_init != init || st.g_init_vec != init_vec ||
                st.g_sched != sched ||
                st.g_order != ctx.pr_order || st.g_tune != ctx.tune_gen) {
                if (st.exec) cudaGraphExecDestroy(st.exec);
                st.exec = nullptr;
                cudaGraph_t gr;
                MB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                try {
                    emit(s);
                } catch (...) {
                    cudaStreamEndCapture(s, &gr);
                    throw;
                }
                MB_CUDA(cudaStreamEndCapture(s, &gr));
                cudaError_t e = cudaGraphInstantiate(&st.exec, gr, 0);
                cudaGraphDestroy(gr);
                MB_CUDA(e);
                st.g_iters = iters;
                st.g_init = init;
                st.g_init_vec = init_vec;
                st.g_sched = sched;
                st.g_order = ctx.pr_order;
                st.g_tune = ctx.tune_gen;
            }
            MB_CUDA(cudaEventRecord(e0, s));
            MB_CUDA(cudaGraphLaunch(st.exec, s));
            MB_CUDA(cudaEventRecord(e1, s));
        } else {
            MB_CUDA(cudaEventRecord(e0, s));
            emit(s);
            MB_CUDA(cudaEventRecord(e1, s));
        }
        MB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        MB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (stats) {
            *stats = mb_stats{};
            stats->supersteps = iters;
            stats->edges_traversed = (int64_t)iters * g.E;
            stats->vertices_reached = g.V;
            stats->device_ms = ms;
            stats->schedule_count[unfused ? MB_SCHED_PUSH_UNFUSED : MB_SCHED_PUSH_EDGE_QUEUE] = iters;
            stats->edges_scanned = (int64_t)iters * g.E;
            int64_t per_step;
            if (ref_order && unfused) per_step = 2;
            else if (ref_order)
                per_step = (st.x_nhub > 0) + (st.x_nbig > 0) + (st.x_nhub > st.x_nbig) + (st.ngroups > 0) +
                           (st.x_nlight > 0);
            else per_step = (unfused ? 2 : st.nlight > 0) + (st.nitems > 0) + (st.nhub > 0);
            stats->kernel_launches = 1 + (int64_t)iters * per_step + (iters == 0);
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
