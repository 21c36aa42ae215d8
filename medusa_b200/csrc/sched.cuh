// sched.cuh -- the learned superstep scheduler: features and single-warp
// inference of a 6 -> 32 -> 32 -> 8 FP32 MLP (ReLU), run on the device
// between supersteps.  It only picks which schedule (kernel) the next
// superstep runs; every schedule computes identical results.
#pragma once
#include "mb_internal.cuh"

namespace mb {

constexpr int kFeat = 6, kHid = 32, kOut = MB_NUM_SCHEDULES;

// Row-major weights, one contiguous float block (kMlpParams floats).
struct MlpLayout {
    static constexpr int w1 = 0;                    // [kHid][kFeat]
    static constexpr int b1 = w1 + kHid * kFeat;    // [kHid]
    static constexpr int w2 = b1 + kHid;            // [kHid][kHid]
    static constexpr int b2 = w2 + kHid * kHid;     // [kHid]
    static constexpr int w3 = b2 + kHid;            // [kOut][kHid]
    static constexpr int b3 = w3 + kOut * kHid;     // [kOut]
    static constexpr int total = b3 + kOut;
};
constexpr int kMlpParams = MlpLayout::total;

// Scheduler features of a superstep, all roughly in [0, 1]:
//   0 frontier vertices   log2(1+n)/log2(1+V)
//   1 frontier out-edges  log2(1+m)/log2(1+E)
//   2 unvisited vertices  log2(1+nu)/log2(1+V)
//   3 unvisited out-edges log2(1+mu)/log2(1+E)
//   4 degree skew         log2(max out-degree / mean out-degree) / 16
//   5 current frontier format (0 queue, 1 bitmap)
__host__ __device__ inline void make_features(float *f, float n, float m, float nu, float mu,
                                              float V, float E, float skew, int mode) {
    const float lv = log2f(1.0f + V), le = log2f(1.0f + E);
    f[0] = log2f(1.0f + n) / lv;
    f[1] = le > 0.f ? log2f(1.0f + m) / le : 0.f;
    f[2] = log2f(1.0f + fmaxf(nu, 0.f)) / lv;
    f[3] = le > 0.f ? log2f(1.0f + fmaxf(mu, 0.f)) / le : 0.f;
    f[4] = skew / 16.0f;
    f[5] = (float)mode;
}

// Inference by one full warp; returns the argmax in every lane.  Schedules
// whose bit is clear in `allowed` are never picked.
__device__ inline int mlp_pick_warp(const float *__restrict__ P, const float *f, unsigned allowed) {
    const int lane = threadIdx.x & 31;
    float h1 = P[MlpLayout::b1 + lane];
#pragma unroll
    for (int i = 0; i < kFeat; i++) h1 = fmaf(P[MlpLayout::w1 + lane * kFeat + i], f[i], h1);
    h1 = fmaxf(h1, 0.f);
    float h2 = P[MlpLayout::b2 + lane];
#pragma unroll
    for (int i = 0; i < kHid; i++)
        h2 = fmaf(P[MlpLayout::w2 + lane * kHid + i], __shfl_sync(0xffffffffu, h1, i), h2);
    h2 = fmaxf(h2, 0.f);
    // every lane runs the same shuffles; lanes >= kOut compute a dummy row
    const int r = lane < kOut ? lane : 0;
    float o = P[MlpLayout::b3 + r];
#pragma unroll
    for (int i = 0; i < kHid; i++)
        o = fmaf(P[MlpLayout::w3 + r * kHid + i], __shfl_sync(0xffffffffu, h2, i), o);
    if (lane >= kOut || !((allowed >> lane) & 1u)) o = -3.0e38f;
    int best = lane < kOut ? lane : kOut;
    float bv = o;
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        float ov = __shfl_xor_sync(0xffffffffu, bv, off);
        int ob = __shfl_xor_sync(0xffffffffu, best, off);
        if (ov > bv || (ov == bv && ob < best)) {
            bv = ov;
            best = ob;
        }
    }
    return best >= kOut ? 0 : best;
}

}  // namespace mb
