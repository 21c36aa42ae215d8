// noalloc.cu -- PageRank supersteps that allocate no memory.
//
// Some callers cannot call cudaMalloc.  A host application that reserves the
// GPU's memory for its own pool up front (a database engine or a serving
// process with a fixed memory budget) forbids allocations it did not make,
// and cudaMalloc/cudaFree may synchronise the whole device, which a
// latency-bound caller cannot afford inside a call.  For them,
// mb_pagerank_noalloc takes only device arrays the caller already owns (the
// out-edge offsets, the in-edge offsets and in-edge sources, and the output
// ranks) and keeps its scratch -- the two contribution buffers rank/outdeg of
// consecutive supersteps -- in one fixed file-scope device array,
// g_pr_scratch, which every GPU that loads this library holds until the
// process exits.  Graphs with more than kNoAllocMaxVertices vertices are
// rejected.
//
// The arithmetic is the same as mb_pagerank's (the order of pr_order.cuh),
// so the two give identical bits.  Heavier vertices' blocks are summed by
// the warp that owns the vertex's 32-vertex group, one vertex after the
// other, instead of by a separate block kernel: the block sums would need
// more scratch.
#include <mutex>
#include "mb_internal.cuh"
#include "pr_order.cuh"

namespace mb {
void record_thread_error(const std::string &msg);  // capi.cu
}

namespace {

constexpr int32_t kNoAllocMaxVertices = 1 << 20;  // 2 x 4 MiB of scratch
constexpr int kNaWin = 1024;
constexpr int kNaWarps = 8;
constexpr int kMaxDevices = 64;

// Scratch shared by every call on a device: contribution buffers 0 and 1.
// Every element a call reads is written earlier in the same call, so nothing
// has to be cleared between calls.
__device__ __align__(256) float g_pr_scratch[2 * kNoAllocMaxVertices];

struct NaArgs {
    int32_t V;
    const int32_t *row, *rrow, *rcol;
    const float *cin;
    float *cout;
    float *rank;
};

__device__ __forceinline__ int32_t na_outdeg(const NaArgs &a, int32_t v) {
    return a.row[v + 1] - a.row[v];
}

__device__ __forceinline__ void na_write(const NaArgs &a, int32_t v, float sum) {
    const float r = mb::pr_update(sum);
    a.rank[v] = r;
    const int32_t d = na_outdeg(a, v);
    a.cout[v] = d > 0 ? r / (float)d : 0.0f;
}

__global__ void k_na_init(const int32_t *row, int32_t V, float init, float *c) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < V;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = row[u + 1] - row[u];
        c[u] = d > 0 ? init / (float)d : 0.0f;
    }
}

__global__ void k_na_fill(float *x, int32_t n, float v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] = v;
}

// One warp per 32 consecutive vertices, light in-edge lists streamed through
// a shared window; then the warp sums each heavier vertex's blocks in turn.
__global__ void __launch_bounds__(kNaWarps * 32) k_na_pull(NaArgs a) {
    __shared__ float win[kNaWarps][kNaWin];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float *wv = win[wid];
    const int64_t ngroups = ((int64_t)a.V + 31) / 32;
    for (int64_t grp = (int64_t)blockIdx.x * kNaWarps + wid; grp < ngroups;
         grp += (int64_t)gridDim.x * kNaWarps) {
        const int32_t v = (int32_t)(grp * 32 + lane);
        const bool valid = v < a.V;
        const int32_t vb = (int32_t)(grp * 32);
        const int32_t ve = (int32_t)min(grp * 32 + 32, (int64_t)a.V);
        int64_t b = 0, e = 0;
        if (valid) {
            b = a.rrow[v];
            e = a.rrow[v + 1];
        }
        const bool hub = valid && (e - b) > mb::kPrLight;
        const int64_t g0 = a.rrow[vb], g1 = a.rrow[ve];
        float sum = 0.f;
        for (int64_t w0 = g0; w0 < g1; w0 += kNaWin) {
            const int64_t w1 = min(w0 + (int64_t)kNaWin, g1);
            const bool mine = !hub && b < w1 && e > w0;
            if (!__any_sync(0xffffffffu, mine)) continue;
            for (int k = lane; k < kNaWin; k += 32) {
                const int64_t j = w0 + k;
                if (j < w1) wv[k] = __ldg(&a.cin[a.rcol[j]]);
            }
            __syncwarp();
            if (mine) {
                const int64_t lo = max(b, w0), hi = min(e, w1);
                for (int64_t j = lo; j < hi; j++) sum += wv[j - w0];
            }
            __syncwarp();
        }
        for (unsigned hm = __ballot_sync(0xffffffffu, hub); hm; hm &= hm - 1) {
            const int owner = __ffs(hm) - 1;
            const int64_t hb = __shfl_sync(0xffffffffu, b, owner);
            const int64_t he = __shfl_sync(0xffffffffu, e, owner);
            float tot = 0.f;
            for (int64_t j0 = hb; j0 < he; j0 += mb::kPrBlock) {
                const int64_t j1 = min(he, j0 + (int64_t)mb::kPrBlock);
                tot += mb::pr_warp_block_sum(j0, j1, [&](int64_t j) { return __ldg(&a.cin[a.rcol[j]]); });
            }
            if (lane == owner) sum = tot;
        }
        if (valid) na_write(a, v, sum);
    }
}

std::mutex g_mu;
int g_num_sms[kMaxDevices];

// Device memory of device `dev` (or managed memory, which every device
// reaches).  Device memory of another GPU is refused: without peer access
// the kernels would fault on it.
bool is_device_memory(const void *p, int dev) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == dev;
}

int na_fail(int code, const std::string &msg) {
    mb::record_thread_error("mb_pagerank_noalloc: " + msg);
    return code;
}

}  // namespace

extern "C" int mb_pagerank_noalloc(const int32_t *row, const int32_t *rrow, const int32_t *rcol,
                                   int32_t num_vertices, int64_t num_edges, int32_t iters,
                                   float init, float *rank_out, void *stream) {
    const int32_t V = num_vertices;
    if (V < 1) return na_fail(MB_ERR_INVALID, "num_vertices must be >= 1");
    if (V > kNoAllocMaxVertices)
        return na_fail(MB_ERR_UNSUPPORTED, "num_vertices " + std::to_string(V) +
                                               " exceeds the no-allocation scratch limit of " +
                                               std::to_string(kNoAllocMaxVertices));
    if (num_edges < 0 || num_edges > 0x7FFFFFFFll) return na_fail(MB_ERR_INVALID, "bad num_edges");
    if (iters < 0) return na_fail(MB_ERR_INVALID, "iters must be >= 0");
    if (!row || !rrow || !rank_out || (num_edges > 0 && !rcol))
        return na_fail(MB_ERR_INVALID, "null array");
    // an error left pending by the caller's earlier CUDA calls on this thread
    // is cleared here, so that the check after the launches reports only
    // this call's own errors
    cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return na_fail(MB_ERR_CUDA, "no current CUDA device");
    }
    if (!is_device_memory(row, dev) || !is_device_memory(rrow, dev) ||
        !is_device_memory(rank_out, dev) || (num_edges > 0 && !is_device_memory(rcol, dev)))
        return na_fail(MB_ERR_INVALID, "every array must be device memory of the current device");
    // The scratch array's device address in the CURRENT context, looked up
    // on every call (a lookup, no allocation): the host-side name
    // g_pr_scratch is not a device address, and an address cached from an
    // earlier context (before a cudaDeviceReset, or under another context
    // the host made current through the driver API) would be stale.  The
    // first call in a context also loads the library's device code there.
    float *scratch = nullptr;
    {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_pr_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return na_fail(MB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        }
        scratch = (float *)p;
    }
    int sms = 0;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_num_sms[dev]) {
            const cudaError_t e = cudaDeviceGetAttribute(&g_num_sms[dev], cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) {
                cudaGetLastError();
                g_num_sms[dev] = 0;
                return na_fail(MB_ERR_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
            }
        }
        sms = g_num_sms[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    float *c[2] = {scratch, scratch + kNoAllocMaxVertices};
    const int grid = sms * 8;
    if (iters == 0) {
        k_na_fill<<<grid, 256, 0, s>>>(rank_out, V, init);
    } else {
        k_na_init<<<grid, 256, 0, s>>>(row, V, init, c[0]);
        for (int it = 0; it < iters; it++) {
            NaArgs a{V, row, rrow, rcol, c[it & 1], c[(it & 1) ^ 1], rank_out};
            k_na_pull<<<grid, kNaWarps * 32, 0, s>>>(a);
        }
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(MB_ERR_CUDA, cudaGetErrorString(e));
    return MB_OK;
}
