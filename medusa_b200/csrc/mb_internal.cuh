// mb_internal.cuh -- shared internals of libmedusa_b200 (not part of the C ABI).
//
// Device-side layout of a graph (all int32/uint32 SoA arrays in HBM):
//   row[V+1]   CSR offsets of out-edges         (the reference's edge_index,
//                                                SSSP/VertexDataType.cu:79-83)
//   col[E]     destination of each out-edge      (EdgeArray::dstVertexID)
//   esrc[E]    source of each out-edge           (EdgeArray::srcVertexID)
//   wt[E]      float weight of each out-edge     (EdgeArray::weight)
//   rrow[V+1]  CSC offsets of in-edges           (VertexArray::msg_index,
//                                                SSSP/VertexDataType.cu:75-77)
//   rcol[E]    source of each in-edge, grouped by destination
//   rwt[E]     weight of each in-edge
//   mslot[E]   CSC position of CSR edge e        (EdgeArray::msgDstID,
//                                                SSSP/EdgeDataType.cu:181-182)
// Out-edges of a vertex keep the reference's AA order when the graph is built
// with MB_ORDER_REFERENCE; in-edges of a vertex are in CSR order (a stable
// sort), which is exactly the order the reference's msgDstID assigns.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "../../include/medusa_b200.h"

namespace mb {

constexpr int kWarp = 32;
constexpr float kMedusaMax = 1000000000.0f;  // SSSP/Configuration.h:6

struct CudaError {
    cudaError_t err;
    const char *what;
    const char *file;
    int line;
};

#define MB_CUDA(call)                                                        \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) throw ::mb::CudaError{e_, #call, __FILE__, __LINE__}; \
    } while (0)

#define MB_CHECK_LAUNCH() MB_CUDA(cudaGetLastError())

struct ApiError {
    int code;
    std::string msg;
};

[[noreturn]] inline void fail(int code, const std::string &msg) { throw ApiError{code, msg}; }

// A device buffer owned by a context or graph.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // grow (never shrink); contents are not preserved
    void *reserve(size_t n) {
        if (n <= bytes && p) return p;
        release();
        size_t want = n < 256 ? 256 : n;
        MB_CUDA(cudaMalloc(&p, want));
        bytes = want;
        return p;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

struct AppStates;  // per-app run state cached on a graph (capi.cu)

struct Graph {
    AppStates *apps = nullptr;
    int32_t V = 0;
    int64_t E = 0;
    bool weighted = false;
    int device = 0;
    DevBuf row, col, esrc, wt, rrow, rcol, rwt, mslot, outdeg;
    int32_t max_outdeg = 0, max_indeg = 0;
    void release() {
        row.release(); col.release(); esrc.release(); wt.release();
        rrow.release(); rcol.release(); rwt.release(); mslot.release(); outdeg.release();
    }
};

struct Context;

// ---- device-wide primitives (prim.cu) -------------------------------------
// Exclusive prefix sum of n uint32 values into out (may alias in); the total
// goes to *total_dev when non-null.  Scratch comes from ctx.
void scan_exclusive_u32(Context &ctx, const uint32_t *in, uint32_t *out, int64_t n,
                        uint32_t *total_dev, cudaStream_t s);
// Stable LSD radix sort of (key,value) pairs by the low `bits` bits of key.
// keys/vals are sorted in place (ping-ponging through ctx scratch).
void radix_sort_pairs(Context &ctx, uint32_t *keys, uint32_t *vals, int64_t n, int bits,
                      cudaStream_t s);

// ---- graph construction (graph.cu) ------------------------------------------
void graph_build_from_device_edges(Context &ctx, Graph &g, int32_t V, int64_t E,
                                   uint32_t *d_src, uint32_t *d_dst, float *d_w,
                                   uint32_t flags);
// A caller's CSR (row checked on the host) -> graph; each row keeps its
// order.  d_col is used as scratch.
void graph_build_from_device_csr(Context &ctx, Graph &g, int32_t V, int64_t E, const int32_t *d_row,
                                 uint32_t *d_col, float *d_w);
// GTgraph text (host or device bytes) -> graph (gtgraph.cu).
void graph_from_gtgraph(Context &ctx, Graph &g, const char *text, int64_t len, uint32_t flags);

// ---- context ------------------------------------------------------------------
struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    std::string last_error;
    // scratch buffers, grown on demand
    DevBuf scratch[8];
    // learned-scheduler weights (kMlpParams floats each), one model per loop
    // kind: MB_MODEL_BFS, MB_MODEL_BATCHED (batched BFS: push vs pull),
    // MB_MODEL_SSSP.  An untrained model leaves its loops on the fixed rule.
    static constexpr int kModels = 3;
    DevBuf mlp[kModels];
    bool mlp_ready[kModels] = {false, false, false};
    const float *model(int m) const { return mlp_ready[m] ? mlp[m].as<float>() : nullptr; }
    void *pinned = nullptr;        // staging for caller host buffers (grown)
    size_t pinned_bytes = 0;
    char *pinned_small = nullptr;  // fixed 64 KiB: run parameters + control readback
    static constexpr size_t kParamsOff = 0, kCtrlOff = 16384, kSmallBytes = 65536;
    int schedule_policy = MB_POLICY_FIXED;
    int fixed_schedule = -1;
    std::vector<int8_t> replay;    // MB_POLICY_ORACLE_BEST schedule list
    bool use_graphs = true;
    float sssp_delta = 0.f;        // near-far bucket width (0: off); < 0: chosen per graph
    bool tail = true;              // persistent single-CTA tail for small frontiers
    bool persist = false;          // persistent cooperative grid for schedules 0/4
    bool batching = true;          // several BFS sources: one masked traversal per 64
    bool replay_then_fixed = false;  // replay policy: fixed rule after the list
    int32_t max_step = -1;           // >= 0: runs stop after this superstep
    int pr_order = MB_PR_ORDER_REFERENCE;  // PageRank summation order
    // launch and routing parameters (MB_TUNE_*); -1: the built-in default
    int64_t tunable[MB_NUM_TUNABLES] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                                       -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    uint64_t tune_gen = 0;  // bumped on every change (loop graphs are rebuilt)
    int blocks_per_sm(int which, int dflt) const {
        return tunable[which] > 0 ? (int)tunable[which] : dflt;
    }
    // superstep trace (host-loop runs): one record per superstep
    bool tracing = false;
    struct TraceRec {
        int32_t app, step, sched, branch;
        float feat[8];
        float ms;
        uint32_t n;  // frontier vertices and out-edges the superstep started from
        uint64_t m;
    };
    std::vector<TraceRec> trace;
    void *ctrl_readback() { return pinned_small + kCtrlOff; }
    void *pinned_reserve(size_t n) {
        if (n <= pinned_bytes && pinned) return pinned;
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        MB_CUDA(cudaMallocHost(&pinned, n));
        pinned_bytes = n;
        return pinned;
    }
};

// Superstep cap of a loop: the MB_TUNE_STEP_CAP tunable when set, else the
// loop's own bound; past it a run stops with MB_ERR_TIMEOUT.
inline int step_cap(const Context &ctx, int64_t dflt) {
    const int64_t t = ctx.tunable[MB_TUNE_STEP_CAP];
    return (int)std::min<int64_t>(t >= 0 ? t : dflt, 1 << 30);
}

// Blocking copy ordered with the library's stream.  The stream is
// non-blocking, so a plain cudaMemcpy (legacy default stream) is not ordered
// with it, and a host-to-device cudaMemcpy from pageable memory may return
// before its data has landed: a kernel queued next on the stream could read
// the buffer early.  Every copy into a buffer that the stream's kernels read,
// or out of one they write, goes through here.
inline void copy_sync(cudaStream_t s, void *dst, const void *src, size_t n) {
    if (!n) return;
    MB_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDefault, s));
    MB_CUDA(cudaStreamSynchronize(s));
}

// Pointer classification for the C ABI: device pointers are used in place,
// anything else is treated as host memory and staged.
inline bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

inline int grid_for(int64_t n, int block, int max_blocks) {
    int64_t b = (n + block - 1) / block;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (int)b;
}

// ---- hashing shared by host and device generators --------------------------
__host__ __device__ inline uint64_t mix64(uint64_t z) {
    // SplitMix64 finaliser (Steele, Lea & Flood, OOPSLA 2014)
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ inline uint64_t hash2(uint64_t seed, uint64_t i) {
    return mix64(seed ^ mix64(i));
}
__host__ __device__ inline uint32_t mulhi32(uint32_t r, uint32_t n) {
    return (uint32_t)(((uint64_t)r * (uint64_t)n) >> 32);
}

}  // namespace mb
