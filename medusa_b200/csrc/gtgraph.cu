// gtgraph.cu -- GTgraph text ingest on the GPU.
//
// The reference's only on-disk graph format is GTgraph text, read line by
// line on the host by GTGraph::get_parition (MultipleGPU/PartitionManager.cu
// :153-213): lines up to the first one starting with 'p' are skipped, "p
// <kind> V E" gives the vertex count, then every line starting with 'a' is
// "a <src> <dst> <weight>" with 1-based ids, added in file order.  Here the
// bytes go to the device once and are parsed in parallel:
//   0. the first line that starts with 'p' (atomicMin over line starts);
//   1. every 4096-byte chunk counts the lines after it that start with 'a';
//   2. an exclusive scan of the counts gives each chunk its first edge index;
//   3. every chunk writes its 'a' line starts in order (block scan);
//   4. one thread per edge line parses its three numbers;
// one thread parses the 'p' line.  Edge k is the k-th 'a' line after the
// 'p' line, so the graph built from the parsed arrays equals the
// reference's (AddEdge order).
#include <algorithm>
#include "mb_internal.cuh"

namespace mb {

namespace {

constexpr int kChunk = 4096;
constexpr int kChunkThreads = 256;
constexpr int kPerThread = kChunk / kChunkThreads;

__device__ __forceinline__ bool line_start(const char *t, int64_t i) {
    return i == 0 || t[i - 1] == '\n';
}

// The first line that starts with 'p'.
__global__ void k_find_p(const char *t, int64_t len, unsigned long long *p_pos) {
    const int64_t c0 = (int64_t)blockIdx.x * kChunk;
    for (int k = 0; k < kPerThread; k++) {
        const int64_t i = c0 + (int64_t)threadIdx.x * kPerThread + k;
        if (i < len && t[i] == 'p' && line_start(t, i)) atomicMin(p_pos, (unsigned long long)i);
    }
}

// Lines after the 'p' line that start with 'a' (the reference skips every
// line up to and including the 'p' line).
__device__ __forceinline__ bool edge_line(const char *t, int64_t len, int64_t i, unsigned long long p) {
    return i < len && (unsigned long long)i > p && t[i] == 'a' && line_start(t, i);
}

__global__ void k_count_a(const char *t, int64_t len, uint32_t *cnt, const unsigned long long *p_pos) {
    const int64_t c0 = (int64_t)blockIdx.x * kChunk;
    const unsigned long long p = *p_pos;
    uint32_t n = 0;
    for (int k = 0; k < kPerThread; k++) {
        const int64_t i = c0 + (int64_t)threadIdx.x * kPerThread + k;
        n += edge_line(t, len, i, p);
    }
    __shared__ uint32_t s[kChunkThreads / 32];
    n = __reduce_add_sync(0xffffffffu, n);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int w = 0; w < kChunkThreads / 32; w++) tot += s[w];
        cnt[blockIdx.x] = tot;
    }
}

// Each chunk writes the start offsets of its 'a' lines, in file order.
__global__ void k_write_a(const char *t, int64_t len, const uint32_t *first,
                          const unsigned long long *p_pos, int64_t *starts) {
    const int64_t c0 = (int64_t)blockIdx.x * kChunk;
    const unsigned long long p = *p_pos;
    uint32_t n = 0;
    for (int k = 0; k < kPerThread; k++) {
        const int64_t i = c0 + (int64_t)threadIdx.x * kPerThread + k;
        n += edge_line(t, len, i, p);
    }
    // exclusive block scan of n (thread order = byte order)
    __shared__ uint32_t s[kChunkThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t incl = n;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) s[w] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int k = 0; k < w; k++) before += s[k];
    uint32_t pos = first[blockIdx.x] + before + incl - n;
    for (int k = 0; k < kPerThread; k++) {
        const int64_t i = c0 + (int64_t)threadIdx.x * kPerThread + k;
        if (edge_line(t, len, i, p)) starts[pos++] = i;
    }
}

__device__ __forceinline__ bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// A non-negative or negative integer; false if no digit.
__device__ bool parse_int(const char *t, int64_t len, int64_t &i, int64_t &out) {
    while (i < len && is_space(t[i])) i++;
    bool neg = false;
    if (i < len && (t[i] == '-' || t[i] == '+')) neg = t[i++] == '-';
    int64_t v = 0;
    int digits = 0;
    while (i < len && t[i] >= '0' && t[i] <= '9' && digits < 18) {
        v = v * 10 + (t[i++] - '0');
        digits++;
    }
    if (!digits) return false;
    out = neg ? -v : v;
    return true;
}

// A decimal number: [sign] digits [. digits] [e|E [sign] digits], to float
// through one double (exact for integers below 2^53 and for short
// decimals such as 1.5).
__device__ bool parse_real(const char *t, int64_t len, int64_t &i, float &out) {
    while (i < len && is_space(t[i])) i++;
    bool neg = false;
    if (i < len && (t[i] == '-' || t[i] == '+')) neg = t[i++] == '-';
    unsigned long long mant = 0;
    int sig = 0, scale = 0;
    bool any = false;
    while (i < len && t[i] >= '0' && t[i] <= '9') {
        any = true;
        if (sig < 18) {
            mant = mant * 10 + (unsigned)(t[i] - '0');
            if (mant) sig++;
        } else {
            scale++;
        }
        i++;
    }
    if (i < len && t[i] == '.') {
        i++;
        while (i < len && t[i] >= '0' && t[i] <= '9') {
            any = true;
            if (sig < 18) {
                mant = mant * 10 + (unsigned)(t[i] - '0');
                if (mant) sig++;
                scale--;
            }
            i++;
        }
    }
    if (!any) return false;
    if (i < len && (t[i] == 'e' || t[i] == 'E')) {
        int64_t j = i + 1, ex = 0;
        if (parse_int(t, len, j, ex)) {
            scale += (int)max((int64_t)-400, min((int64_t)400, ex));
            i = j;
        }
    }
    double v = (double)mant;
    if (scale > 0) v *= pow(10.0, (double)scale);
    else if (scale < 0) v /= pow(10.0, (double)-scale);
    out = (float)(neg ? -v : v);
    return true;
}

// One thread per edge line: "a src dst weight" (1-based ids).
__global__ void k_parse_a(const char *t, int64_t len, const int64_t *starts, int64_t E,
                          uint32_t *src, uint32_t *dst, float *w, unsigned *bad) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < E;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = starts[k] + 1, u = 0, v = 0;
        float x = 0.f;
        const bool ok = parse_int(t, len, i, u) && parse_int(t, len, i, v) && parse_real(t, len, i, x);
        if (!ok) atomicOr(bad, 1u);
        // 1-based -> 0-based; out-of-range ids are caught by the graph builder
        src[k] = (uint32_t)(u - 1);
        dst[k] = (uint32_t)(v - 1);
        if (w) w[k] = x;
    }
}

// The 'p' line: "p <kind> V E" -> V.
__global__ void k_parse_p(const char *t, int64_t len, const unsigned long long *p_pos, int64_t *out) {
    out[0] = -1;
    if (*p_pos == ~0ull) return;
    int64_t i = (int64_t)*p_pos + 1;
    while (i < len && is_space(t[i])) i++;
    while (i < len && !is_space(t[i]) && t[i] != '\n') i++;  // the kind word
    int64_t v = 0, e = 0;
    if (parse_int(t, len, i, v)) out[0] = v;
    if (parse_int(t, len, i, e)) out[1] = e;
}

}  // namespace

void graph_from_gtgraph(Context &ctx, Graph &g, const char *text, int64_t len, uint32_t flags) {
    cudaStream_t s = ctx.stream;
    if (len < 0) fail(MB_ERR_INVALID, "negative text length");
    if (len > 0x7FFFFFFFll * 4) fail(MB_ERR_UNSUPPORTED, "GTgraph text larger than 8 GiB");
    DevBuf tb, cnt, first, starts, misc, bs, bd, bw;
    const char *t = text;
    if (!is_device_ptr(text)) {
        t = (const char *)tb.reserve((size_t)std::max<int64_t>(len, 1));
        if (len) MB_CUDA(cudaMemcpyAsync(tb.p, text, (size_t)len, cudaMemcpyHostToDevice, s));
    }
    const int64_t chunks = std::max<int64_t>(1, (len + kChunk - 1) / kChunk);
    if (chunks > 0x7FFFFFFF) fail(MB_ERR_UNSUPPORTED, "GTgraph text too large");
    cnt.reserve(sizeof(uint32_t) * (size_t)chunks);
    first.reserve(sizeof(uint32_t) * (size_t)(chunks + 1));
    misc.reserve(64);
    unsigned long long *p_pos = misc.as<unsigned long long>();        // [0]
    int64_t *pv = (int64_t *)(misc.as<char>() + 8);                    // [1..2] V, E
    uint32_t *total = (uint32_t *)(misc.as<char>() + 24);              // edge lines
    unsigned *bad = (unsigned *)(misc.as<char>() + 28);
    MB_CUDA(cudaMemsetAsync(misc.p, 0xff, 8, s));
    MB_CUDA(cudaMemsetAsync(misc.as<char>() + 8, 0, 56, s));
    if (len > 0) {
        k_find_p<<<(unsigned)chunks, kChunkThreads, 0, s>>>(t, len, p_pos);
        k_count_a<<<(unsigned)chunks, kChunkThreads, 0, s>>>(t, len, cnt.as<uint32_t>(), p_pos);
        MB_CHECK_LAUNCH();
    } else {
        MB_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(uint32_t), s));
    }
    scan_exclusive_u32(ctx, cnt.as<uint32_t>(), first.as<uint32_t>(), chunks, total, s);
    k_parse_p<<<1, 1, 0, s>>>(t, len, p_pos, pv);
    MB_CHECK_LAUNCH();
    int64_t hv[2];
    uint32_t E32 = 0;
    MB_CUDA(cudaMemcpyAsync(hv, pv, sizeof(hv), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaMemcpyAsync(&E32, total, sizeof(E32), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    if (hv[0] < 0) fail(MB_ERR_INVALID, "GTgraph: no 'p <kind> V E' line");
    if (hv[0] < 1 || hv[0] > 0x7FFFFFFFll) fail(MB_ERR_UNSUPPORTED, "GTgraph: vertex count out of range");
    const int64_t E = E32;
    starts.reserve(sizeof(int64_t) * (size_t)std::max<int64_t>(E, 1));
    const size_t eb = sizeof(uint32_t) * (size_t)std::max<int64_t>(E, 1);
    bs.reserve(eb);
    bd.reserve(eb);
    bw.reserve(eb);
    if (E > 0) {
        k_write_a<<<(unsigned)chunks, kChunkThreads, 0, s>>>(t, len, first.as<uint32_t>(), p_pos,
                                                             starts.as<int64_t>());
        k_parse_a<<<grid_for(E, 256, ctx.num_sms * 16), 256, 0, s>>>(t, len, starts.as<int64_t>(), E,
                                                                     bs.as<uint32_t>(), bd.as<uint32_t>(),
                                                                     bw.as<float>(), bad);
        MB_CHECK_LAUNCH();
        unsigned hb = 0;
        MB_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        if (hb) fail(MB_ERR_INVALID, "GTgraph: an 'a' line does not hold three numbers");
    }
    tb.release();
    starts.release();
    graph_build_from_device_edges(ctx, g, (int32_t)hv[0], E, bs.as<uint32_t>(), bd.as<uint32_t>(),
                                  bw.as<float>(), flags);
}

}  // namespace mb
