// pr_order.cuh -- PageRank's fixed summation order, shared by every
// PageRank kernel (the fused pull, the reference-structured split and the
// no-allocation entry point), so all of them give identical bits.
//
//   in-degree <= kPrLight: a sequential fold (from 0) over the in-edges in
//     reverse-CSR order -- the order the reference's msgDstID hands out
//     message slots (SSSP/EdgeDataType.cu:181-182), i.e. the sequential CPU
//     sum of MPG/CPUFunctorHoster.cpp:21-26;
//   larger in-degrees: consecutive blocks of kPrBlock in-edges; a block is
//     summed by one warp (lane l folds edges l, l+32, ... of the block in
//     order, then an xor butterfly, whose result is bit-identical in every
//     lane), and the block sums are folded sequentially.
// Update (MPG/UserOperators.h:22-23): "msg_sum *= 0.85" is a double multiply
// rounded to float, "0.15 + msg_sum" a double add rounded to float.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mb {

constexpr int kPrLight = 64;
constexpr int kPrBlock = 4096;

__device__ __forceinline__ float pr_update(float sum) {
    const float s = (float)((double)sum * 0.85);
    return (float)(0.15 + (double)s);
}

// Block sum by a full warp over j in [j0, j1), j1 - j0 <= kPrBlock; val(j)
// gives edge j's message.  Same value in every lane.
template <class F>
__device__ __forceinline__ float pr_warp_block_sum(int64_t j0, int64_t j1, F val) {
    const int lane = threadIdx.x & 31;
    float s = 0.f;
#pragma unroll 8
    for (int64_t j = j0 + lane; j < j1; j += 32) s += val(j);
#pragma unroll
    for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    return s;
}

// ---- the reference's sequential sum, computed in parallel -------------------
// The reference folds a vertex's messages one after another in float
// (MPG/CPUFunctorHoster.cpp:21-26), in its MEG slot order.  Messages are
// non-negative, so the running sum s never decreases.  While s stays in one
// binade [2^e, 2^(e+1)), every float there is an integer multiple of u =
// ulp(s) and fl(s + x) = s + u * round(x / u), except when x / u ends in
// exactly one half (a tie: rounded to even, i.e. by s's last bit).  A run of
// additions that neither leaves the binade nor meets a tie is therefore s
// plus u times an INTEGER sum, which threads can form in any order.  The
// kernels scan those integers in parallel; the first thread whose prefix
// reaches the binade's end (2^24 units) or that holds a tie folds its own
// elements with float adds from the exact running sum, and the threads after
// it rescan in the new binade.  Binade crossings grow like log2(in-degree),
// so nearly every chunk costs one scan.  Any input the integer path cannot
// take (a term larger than s, a zero or non-finite s, a negative term) lands
// on the float path, which is the reference's own arithmetic.

// round(x / u) for u the ulp of a float with biased exponent ks, clamped to
// 2^23 (any value that large already ends the binade), and whether x / u
// ends in exactly one half.
__device__ __forceinline__ uint32_t pr_units(float x, uint32_t ks, bool &tie) {
    const uint32_t bx = __float_as_uint(x);
    uint32_t ex = bx >> 23;
    uint32_t m = bx & 0x7fffffu;
    if (ex) m |= 0x800000u;
    else ex = 1;  // zero or subnormal
    const int d = (int)ks - (int)ex;
    if (d < 0) return 1u << 23;
    if (d == 0) return min(m, 1u << 23);
    if (d > 24) return 0u;  // x < u / 2
    const uint32_t r = m & ((1u << d) - 1u), h = 1u << (d - 1);
    tie |= (r == h);
    return (m >> d) + (r > h ? 1u : 0u);
}

// The float with biased exponent ks and 24-bit significand b (2^23 <= b < 2^24).
__device__ __forceinline__ float pr_make(uint32_t ks, uint32_t b) {
    return __uint_as_float((ks << 23) | (b & 0x7fffffu));
}

}  // namespace mb
