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
// them independent and coalesced: lane j holds column j of each weight row,
// and a row's dot product with the previous layer (lane j holding unit j)
// is a warp all-reduce.  ~50 loads per lane in flight at once, then ~40
// butterfly reductions.
__device__ __forceinline__ float warp_allsum_f(float x) {
#pragma unroll
    for (int off = 16; off; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    return x;
}

// The MLP's weights as one warp holds them (per lane: column `lane` of
// every weight row, its own biases).
struct MlpRegs {
    float w1r[kFeat], w2r[kHid], w3r[kOut];
    float bias1, bias2, bias3;
    float lo, hi;  // lane i < kFeat: training range of feature i
};

// Issue every weight load (independent, coalesced); callers start this
// before other work so the loads' latency overlaps it.
__device__ __forceinline__ void mlp_load_warp(const float *__restrict__ P, MlpRegs &r) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < kFeat; i++) r.w1r[i] = __ldg(&P[MlpLayout::w1 + lane * kFeat + i]);
#pragma unroll
    for (int i = 0; i < kHid; i++) r.w2r[i] = __ldg(&P[MlpLayout::w2 + i * kHid + lane]);
#pragma unroll
    for (int k = 0; k < kOut; k++) r.w3r[k] = __ldg(&P[MlpLayout::w3 + k * kHid + lane]);
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
    // layer 2: unit i = sum over lanes j of w2[i][j] * h1[j]; lane i keeps it
    float h2 = 0.f;
#pragma unroll
    for (int i = 0; i < kHid; i++) {
        const float sum = warp_allsum_f(r.w2r[i] * h1);
        if (lane == i) h2 = sum;
    }
    h2 = fmaxf(h2 + r.bias2, 0.f);
    float o = 0.f;
#pragma unroll
    for (int k = 0; k < kOut; k++) {
        const float sum = warp_allsum_f(r.w3r[k] * h2);
        if (lane == k) o = sum;
    }
    o += r.bias3;
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
