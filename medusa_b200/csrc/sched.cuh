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
// A model's device block: the parameters, then the per-feature range of its
// training set (lo[kFeat], hi[kFeat]) -- inside a run the network may
// override the fixed rule only on features inside that range.
constexpr int kBoundsOff = kMlpParams;
constexpr int kModelFloats = kMlpParams + 2 * kFeat;
constexpr float kBoundsSlack = 1.0f / 32.0f;  // one doubling of any count

// Scheduler features of a superstep, all in [0, 1].  Counts are absolute
// (log2 / 32), not relative to the graph: whether a superstep is latency- or
// bandwidth-bound depends on its absolute size, and ratios such as
// frontier edges / unvisited edges are differences of these logs.
//   0 frontier vertices   log2(1+n)/32
//   1 frontier out-edges  log2(1+m)/32
//   2 unvisited vertices  log2(1+nu)/32
//   3 unvisited out-edges log2(1+mu)/32
//   4 degree skew         log2(max out-degree / mean out-degree) / 16
//   5 current frontier format (0 queue, 1 bitmap)
__host__ __device__ inline void make_features(float *f, float n, float m, float nu, float mu,
                                              float V, float E, float skew, int mode) {
    (void)V;
    (void)E;
    f[0] = log2f(1.0f + n) * (1.0f / 32.0f);
    f[1] = log2f(1.0f + m) * (1.0f / 32.0f);
    f[2] = log2f(1.0f + fmaxf(nu, 0.f)) * (1.0f / 32.0f);
    f[3] = log2f(1.0f + fmaxf(mu, 0.f)) * (1.0f / 32.0f);
    f[4] = fminf(skew, 16.0f) / 16.0f;
    f[5] = (float)mode;
}

// Inference by one full warp; returns the argmax in every lane.  Schedules
// whose bit is clear in `allowed` are never picked.  Latency matters (it
// runs between supersteps), so every weight load is issued first, all of
// them independent: lane i holds row i of W1 and W2 and row i mod 8 of W3
// (16-byte loads), and computes unit i from the previous layer's units,
// which arrive by one shuffle each -- 32 shuffles and FMAs per layer instead
// of a 5-step all-reduce per unit.
// The MLP's weights as one warp holds them (per lane i: row i of W1 and W2,
// row i mod kOut of W3, its own biases).
struct MlpRegs {
    float w1r[kFeat], w2r[kHid], w3r[kHid];
    float bias1, bias2, bias3;
    float lo, hi;  // lane i < kFeat: training range of feature i
};
static_assert(MlpLayout::w2 % 4 == 0 && MlpLayout::w3 % 4 == 0 && kHid % 4 == 0,
              "W2 and W3 rows are read as float4");

// Issue every weight load (independent, coalesced); callers start this
// before other work so the loads' latency overlaps it.
__device__ __forceinline__ void mlp_load_warp(const float *__restrict__ P, MlpRegs &r) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < kFeat; i++) r.w1r[i] = __ldg(&P[MlpLayout::w1 + lane * kFeat + i]);
    const float4 *w2 = reinterpret_cast<const float4 *>(P + MlpLayout::w2 + lane * kHid);
    const float4 *w3 = reinterpret_cast<const float4 *>(P + MlpLayout::w3 + (lane % kOut) * kHid);
#pragma unroll
    for (int q = 0; q < kHid / 4; q++) {
        const float4 x = __ldg(&w2[q]), y = __ldg(&w3[q]);
        r.w2r[4 * q] = x.x;
        r.w2r[4 * q + 1] = x.y;
        r.w2r[4 * q + 2] = x.z;
        r.w2r[4 * q + 3] = x.w;
        r.w3r[4 * q] = y.x;
        r.w3r[4 * q + 1] = y.y;
        r.w3r[4 * q + 2] = y.z;
        r.w3r[4 * q + 3] = y.w;
    }
    r.bias1 = __ldg(&P[MlpLayout::b1 + lane]);
    r.bias2 = __ldg(&P[MlpLayout::b2 + lane]);
    r.bias3 = __ldg(&P[MlpLayout::b3 + (lane < kOut ? lane : 0)]);
    r.lo = __ldg(&P[kBoundsOff + (lane < kFeat ? lane : 0)]);
    r.hi = __ldg(&P[kBoundsOff + kFeat + (lane < kFeat ? lane : 0)]);
}

// The decision of one full warp (same value in every lane).  Among the
// schedules whose bit is set in `allowed`, the one with the largest output;
// with a fallback schedule (>= 0, allowed), that one is kept unless every
// feature lies within the training range (+- kBoundsSlack) and the best
// output beats the fallback's by more than `margin` (logits): the fixed rule
// stays in charge where the network has not seen such a superstep or is not
// clearly better.
__device__ inline int mlp_decide_warp(const MlpRegs &r, const float *f, unsigned allowed,
                                      int fallback, float margin) {
    const int lane = threadIdx.x & 31;
    float h1 = r.bias1;
#pragma unroll
    for (int i = 0; i < kFeat; i++) h1 = fmaf(r.w1r[i], f[i], h1);
    h1 = fmaxf(h1, 0.f);
    // layer 2: lane i computes unit i = sum_j w2[i][j] * h1[j], h1[j] from
    // lane j (two accumulators halve the dependent FMA chain)
    float s0 = r.bias2, s1 = 0.f;
#pragma unroll
    for (int j = 0; j < kHid; j += 2) {
        s0 = fmaf(r.w2r[j], __shfl_sync(0xffffffffu, h1, j), s0);
        s1 = fmaf(r.w2r[j + 1], __shfl_sync(0xffffffffu, h1, j + 1), s1);
    }
    const float h2 = fmaxf(s0 + s1, 0.f);
    // layer 3: lane k < kOut computes output k (the other lanes' values are
    // discarded below)
    s0 = r.bias3;
    s1 = 0.f;
#pragma unroll
    for (int j = 0; j < kHid; j += 2) {
        s0 = fmaf(r.w3r[j], __shfl_sync(0xffffffffu, h2, j), s0);
        s1 = fmaf(r.w3r[j + 1], __shfl_sync(0xffffffffu, h2, j + 1), s1);
    }
    float o = s0 + s1;
    const float o_fb = __shfl_sync(0xffffffffu, o, fallback >= 0 ? (fallback & 31) : 0);
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
    if (best >= kOut) best = 0;
    if (fallback >= 0 && fallback < kOut && ((allowed >> fallback) & 1u)) {
        float fl = 0.f;
#pragma unroll
        for (int i = 0; i < kFeat; i++)
            if (lane == i) fl = f[i];
        const bool inside = lane >= kFeat || (fl >= r.lo - kBoundsSlack && fl <= r.hi + kBoundsSlack);
        if (!__all_sync(0xffffffffu, inside) || !(bv - o_fb > margin)) return fallback;
    }
    return best;
}

// Plain argmax (no fallback).
__device__ inline int mlp_pick_warp(const float *__restrict__ P, const float *f, unsigned allowed) {
    MlpRegs r;
    mlp_load_warp(P, r);
    return mlp_decide_warp(r, f, allowed, -1, 0.f);
}

// Logit margin by which the network must beat the fixed rule's choice to
// override it inside a run.
constexpr float kOverrideMargin = 1.0f;

}  // namespace mb
