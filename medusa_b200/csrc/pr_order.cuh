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

}  // namespace mb
