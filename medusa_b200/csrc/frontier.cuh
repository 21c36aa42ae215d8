// frontier.cuh -- frontier queue / bitmap building blocks shared by the BFS
// and SSSP superstep kernels.
//
// Queue frontier.  Entry i holds a vertex qv[i] and qo[i], the exclusive
// prefix sum of out-degrees over entries 0..i-1.  Producers reserve
// (count, edges) with ONE 64-bit atomicAdd of (n << 32 | sum_deg) per warp,
// so a queue comes out already scanned: the next superstep can split its
// edges evenly across CTAs (merge-path) without a separate scan pass.  For
// the same purpose the producer of an entry also records, for every tile of
// kTile edges whose first edge falls inside that entry's range, the entry's
// index in tile_first[].  Vertices with no out-edges are never queued.
//
// Bitmap frontier.  One bit per vertex in uint32 words; a warp owns a word
// and builds it with __ballot_sync, so pull steps need no atomics.
#pragma once
#include "mb_internal.cuh"

namespace mb {

// Loads that bypass L1: counters other threads update with atomics (at L2)
// are read this way by code that may run inside the same kernel.
template <class T>
__device__ __forceinline__ T ldg2(const T *p) { return __ldcg(p); }


#ifndef MB_TILE_EDGES
#define MB_TILE_EDGES 512
#endif
constexpr int kTile = MB_TILE_EDGES;  // edges per merge-path tile
constexpr int kPushThreads = 256;    // threads per push CTA
constexpr int kTileItems = kTile / kPushThreads;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated enqueue.  Must be called by all 32 lanes of the warp.
// Lanes with pred enqueue (v, deg); deg must be > 0 for those lanes.
__device__ __forceinline__ void enqueue_warp(bool pred, int32_t v, uint32_t deg,
                                             unsigned long long *qctr, int32_t *qv,
                                             uint32_t *qo, int32_t *tile_first) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    uint32_t d = pred ? deg : 0u;
    uint32_t incl = d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader)
        base = atomicAdd(qctr, ((unsigned long long)__popc(mask) << 32) | total);
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) {
        const uint32_t pos = (uint32_t)(base >> 32) + __popc(mask & lanemask_lt());
        const uint32_t off = (uint32_t)base + incl - d;
        qv[pos] = v;
        qo[pos] = off;
        const uint32_t t0 = (off + kTile - 1) / kTile, t1 = (off + d - 1) / kTile;
        for (uint32_t t = t0; t <= t1; t++) tile_first[t] = (int32_t)pos;
    }
}

// CTA-level enqueue buffer: a tile's discoveries are gathered in shared
// memory and published with ONE global atomicAdd per tile (instead of one
// per warp per round on the same counter, which serialises in L2).
// Capacity kTile: a tile has kTile edges and each edge discovers at most one
// vertex.
struct BlockQueue {
    int32_t v[kTile];
    uint32_t d[kTile];
    uint32_t n;
    uint32_t warp_tot[kPushThreads / 32];
    unsigned long long base;
};

// Warp-aggregated append to the block buffer (all 32 lanes call it).
__device__ __forceinline__ void bq_push(BlockQueue &bq, bool pred, int32_t v, uint32_t deg) {
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&bq.n, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) {
        const uint32_t i = base + __popc(mask & lanemask_lt());
        bq.v[i] = v;
        bq.d[i] = deg;
    }
}

// Publish the block buffer to the global queue and reset it (all threads of
// the block call it; it synchronises the block).
__device__ __forceinline__ void bq_flush(BlockQueue &bq, unsigned long long *qctr, int32_t *qv,
                                         uint32_t *qo, int32_t *tile_first) {
    constexpr int kPer = kTile / kPushThreads;
    __syncthreads();
    const uint32_t n = bq.n;
    if (n == 0) return;  // block-uniform
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t i0 = threadIdx.x * kPer;
    uint32_t loc[kPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        loc[k] = (i0 + k < n) ? bq.d[i0 + k] : 0u;
        sum += loc[k];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) bq.warp_tot[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int w = 0; w < kPushThreads / 32; w++) {
            const uint32_t t = bq.warp_tot[w];
            bq.warp_tot[w] = tot;
            tot += t;
        }
        bq.base = atomicAdd(qctr, ((unsigned long long)n << 32) | tot);
    }
    __syncthreads();
    const unsigned long long base = bq.base;
    uint32_t off = (uint32_t)base + bq.warp_tot[wid] + incl - sum;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        const uint32_t i = i0 + k;
        if (i < n) {
            const uint32_t pos = (uint32_t)(base >> 32) + i;
            const uint32_t d = loc[k];
            qv[pos] = bq.v[i];
            qo[pos] = off;
            const uint32_t t0 = (off + kTile - 1) / kTile, t1 = (off + d - 1) / kTile;
            for (uint32_t t = t0; t <= t1; t++) tile_first[t] = (int32_t)pos;
            off += d;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) bq.n = 0;
    __syncthreads();
}

// Index of the last element of s[0..n) that is <= x (s ascending, s[0] <= x).
__device__ __forceinline__ int upper_bound_minus1(const uint32_t *s, int n, uint32_t x) {
    int lo = 0, hi = n;  // answer in [lo, hi)
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (s[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

// x[i] for a two-element parameter array, without dynamic indexing (which
// would copy the kernel parameter array to local memory).
template <class T>
__device__ __forceinline__ T pick(T const (&x)[2], int i) { return i ? x[1] : x[0]; }

__device__ __forceinline__ bool test_bit(const uint32_t *bm, int32_t v) {
    return (bm[v >> 5] >> (v & 31)) & 1u;
}

// Warp-level sum, result in all lanes.
template <class T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

}  // namespace mb
