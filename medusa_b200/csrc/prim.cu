// prim.cu -- device-wide primitives used to build graph storage on the GPU:
// an exclusive prefix sum and a stable LSD radix sort of (key, value) pairs.
//
// These replace the reference's serial host loops that build the CSR and the
// per-destination message slots (SSSP/EdgeDataType.cu:138-186,
// SSSP/VertexDataType.cu:64-85): a stable sort by source gives the CSR, a
// stable sort of the CSR by destination gives the reverse CSR and, through
// its permutation, the reference's msgDstID.
#include "mb_internal.cuh"

namespace mb {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Block-wide exclusive scan of one value per thread; returns the block total
// in *total (all threads).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t *total) {
    __shared__ uint32_t warp_tot[kScanThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = warp_incl_scan(x);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        constexpr int kW = kScanThreads / 32;
        uint32_t t = lane < kW ? warp_tot[lane] : 0;
        uint32_t ti = warp_incl_scan(t);
        if (lane < kW) warp_tot[lane] = ti - t;  // exclusive prefix of warp totals
        if (lane == kW - 1) *total = ti;
    }
    __syncthreads();
    uint32_t r = warp_tot[wid] + inc - x;
    __syncthreads();
    return r;
}

__global__ void k_scan_reduce(const uint32_t *__restrict__ in, int64_t n,
                              uint32_t *__restrict__ partial) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        int64_t j = base + i * kScanThreads + threadIdx.x;
        if (j < n) s += in[j];
    }
    __shared__ uint32_t tot;
    (void)block_excl_scan(s, &tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void k_scan_apply(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                             int64_t n, const uint32_t *__restrict__ partial,
                             uint32_t *__restrict__ total_dev) {
    __shared__ uint32_t sm[kScanTile + kScanTile / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    // striped, coalesced load into padded shared memory
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        int idx = i * kScanThreads + threadIdx.x;
        int64_t j = base + idx;
        sm[idx + (idx >> 5)] = j < n ? in[j] : 0u;
    }
    __syncthreads();
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        int idx = threadIdx.x * kScanItems + i;
        v[i] = sm[idx + (idx >> 5)];
        s += v[i];
    }
    __shared__ uint32_t tot;
    uint32_t run = block_excl_scan(s, &tot) + (partial ? partial[blockIdx.x] : 0u);
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        int idx = threadIdx.x * kScanItems + i;
        sm[idx + (idx >> 5)] = run;
        run += v[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        int idx = i * kScanThreads + threadIdx.x;
        int64_t j = base + idx;
        if (j < n) out[j] = sm[idx + (idx >> 5)];
    }
    if (total_dev && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1)
        *total_dev = run;  // exclusive prefix of the last thread + its items
}

// ---------------------------------------------------------------------------
// radix sort

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096 keys per tile
constexpr int kRadix = 256;

__global__ void k_radix_hist(const uint32_t *__restrict__ keys, int64_t n, int shift,
                             uint32_t *__restrict__ hist, int64_t ntiles) {
    __shared__ uint32_t h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kSortRounds; r++) {
        int64_t j = base + r * kSortThreads + threadIdx.x;
        if (j < n) atomicAdd(&h[(keys[j] >> shift) & 0xff], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void k_radix_scatter(const uint32_t *__restrict__ keys_in,
                                const uint32_t *__restrict__ vals_in,
                                uint32_t *__restrict__ keys_out,
                                uint32_t *__restrict__ vals_out, int64_t n, int shift,
                                const uint32_t *__restrict__ hist_scan, int64_t ntiles) {
    constexpr int kWarps = kSortThreads / 32;
    __shared__ uint32_t base_off[kRadix];
    __shared__ uint32_t run[kRadix];
    __shared__ uint32_t wcnt[kWarps][kRadix];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    base_off[threadIdx.x] = hist_scan[(int64_t)threadIdx.x * ntiles + blockIdx.x];
    run[threadIdx.x] = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kSortRounds; r++) {
        int64_t j = base + r * kSortThreads + threadIdx.x;
        bool valid = j < n;
        uint32_t key = valid ? keys_in[j] : 0u;
        uint32_t val = valid ? vals_in[j] : 0u;
        uint32_t d = valid ? ((key >> shift) & 0xffu) : 0x100u;  // 0x100: no digit
        unsigned peers = __match_any_sync(0xffffffffu, d);
        uint32_t rank = __popc(peers & lt);
        if (valid && rank == 0) wcnt[wid][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t pos = base_off[d] + run[d] + rank;
            for (int w = 0; w < wid; w++) pos += wcnt[w][d];
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
        {
            uint32_t add = 0;
#pragma unroll
            for (int w = 0; w < kWarps; w++) {
                add += wcnt[w][threadIdx.x];
                wcnt[w][threadIdx.x] = 0;
            }
            run[threadIdx.x] += add;
        }
        __syncthreads();
    }
}

}  // namespace

void scan_exclusive_u32(Context &ctx, const uint32_t *in, uint32_t *out, int64_t n,
                        uint32_t *total_dev, cudaStream_t s) {
    if (n <= 0) {
        if (total_dev) MB_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), s));
        return;
    }
    int64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 1) {
        k_scan_apply<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total_dev);
        MB_CHECK_LAUNCH();
        return;
    }
    // partial sums of the tiles live in their own allocation (recursion-safe)
    DevBuf partial;
    partial.reserve(sizeof(uint32_t) * (size_t)nb);
    try {
        k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, partial.as<uint32_t>());
        MB_CHECK_LAUNCH();
        scan_exclusive_u32(ctx, partial.as<uint32_t>(), partial.as<uint32_t>(), nb, nullptr, s);
        k_scan_apply<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, partial.as<uint32_t>(),
                                                           total_dev);
        MB_CHECK_LAUNCH();
        MB_CUDA(cudaStreamSynchronize(s));  // partial is freed on return
    } catch (...) {
        partial.release();
        throw;
    }
    partial.release();
}

void radix_sort_pairs(Context &ctx, uint32_t *keys, uint32_t *vals, int64_t n, int bits,
                      cudaStream_t s) {
    if (n <= 1 || bits <= 0) return;
    int64_t ntiles = (n + kSortTile - 1) / kSortTile;
    DevBuf kb, vb, hist;
    try {
        kb.reserve(sizeof(uint32_t) * (size_t)n);
        vb.reserve(sizeof(uint32_t) * (size_t)n);
        hist.reserve(sizeof(uint32_t) * (size_t)(kRadix * ntiles));
        uint32_t *ki = keys, *vi = vals, *ko = kb.as<uint32_t>(), *vo = vb.as<uint32_t>();
        for (int shift = 0; shift < bits; shift += 8) {
            k_radix_hist<<<(unsigned)ntiles, kSortThreads, 0, s>>>(ki, n, shift,
                                                                 hist.as<uint32_t>(), ntiles);
            MB_CHECK_LAUNCH();
            scan_exclusive_u32(ctx, hist.as<uint32_t>(), hist.as<uint32_t>(), kRadix * ntiles,
                               nullptr, s);
            k_radix_scatter<<<(unsigned)ntiles, kSortThreads, 0, s>>>(
                ki, vi, ko, vo, n, shift, hist.as<uint32_t>(), ntiles);
            MB_CHECK_LAUNCH();
            std::swap(ki, ko);
            std::swap(vi, vo);
        }
        if (ki != keys) {
            MB_CUDA(cudaMemcpyAsync(keys, ki, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
            MB_CUDA(cudaMemcpyAsync(vals, vi, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        }
        MB_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        kb.release(); vb.release(); hist.release();
        throw;
    }
    kb.release(); vb.release(); hist.release();
}

}  // namespace mb
