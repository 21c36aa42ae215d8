// graph.cu -- GraphStorage on the device, and the seeded synthetic generators.
//
// The reference builds its layouts on the host, serially, from linked lists
// (GraphIR::AddEdge, MedusaRT/GraphConverter.cu:180-196; EdgeArray::buildAA,
// SSSP/EdgeDataType.cu:138-186; VertexArray::build,
// SSSP/VertexDataType.cu:64-85) and then copies them to the GPU
// (D_EdgeArray::Fill, SSSP/EdgeDataType.cu:364-391).  Here the edge list goes
// to the device once and every array is built there:
//   1. stable radix sort of (src, edge#) -> CSR order.  With
//      MB_ORDER_REFERENCE the edge numbers are taken in reverse, which puts
//      each source's edges in the reverse of insertion order, as GraphIR's
//      prepend-and-walk does;
//   2. row[] = exclusive scan of out-degrees (the reference's edge_index);
//   3. stable radix sort of (dst, csr#) -> reverse CSR.  Stability keeps the
//      in-edges of each destination in CSR order, which is the order the
//      reference's per-destination cursor hands out message slots in
//      (msgDstID, SSSP/EdgeDataType.cu:181-182); mslot[] is that permutation;
//   4. rrow[] = exclusive scan of in-degrees (the reference's msg_index).
#include <algorithm>
#include <cmath>
#include "mb_internal.cuh"

namespace mb {

// ---------------------------------------------------------------------------
// generators: one pure function per edge, shared by host and device code, so
// that the host copy (for the CPU checker) and the device copy are identical.

constexpr uint64_t kWeightSalt = 0x5851F42D4C957F2Dull;
constexpr uint64_t kShortcutSalt = 0x2545F4914F6CDD1Dull;

struct RmatThresholds {
    uint64_t ta, tab, tabc;  // a, a+b, a+b+c scaled by 2^32
};

inline RmatThresholds rmat_thresholds(double a, double b, double c) {
    auto sc = [](double p) -> uint64_t {
        if (p <= 0) return 0;
        if (p >= 1) return 1ull << 32;
        return (uint64_t)std::llround(p * 4294967296.0);
    };
    return {sc(a), sc(a + b), sc(a + b + c)};
}

__host__ __device__ inline void rmat_edge(uint64_t seed, int scale, uint64_t e,
                                          RmatThresholds t, uint32_t *s, uint32_t *d) {
    uint32_t u = 0, v = 0;
    for (int l = 0; l < scale; l += 2) {
        uint64_t h = hash2(seed, e * 32 + (uint64_t)(l >> 1));
        for (int k = 0; k < 2 && l + k < scale; k++) {
            uint64_t r = k ? (uint32_t)h : (uint32_t)(h >> 32);
            uint32_t bs = r >= t.tab ? 1u : 0u;                          // quadrants c, d
            uint32_t bd = ((r >= t.ta && r < t.tab) || r >= t.tabc) ? 1u : 0u;  // b, d
            u = (u << 1) | bs;
            v = (v << 1) | bd;
        }
    }
    *s = u;
    *d = v;
}

__host__ __device__ inline void uniform_edge(uint64_t seed, uint32_t V, uint64_t e,
                                             uint32_t *s, uint32_t *d) {
    uint64_t h = hash2(seed, e);
    *s = mulhi32((uint32_t)(h >> 32), V);
    *d = mulhi32((uint32_t)h, V);
}

__host__ __device__ inline float int_weight(uint64_t seed, uint64_t e, int32_t wmin,
                                            int32_t wmax) {
    if (wmax <= 0) return 1.0f;
    uint32_t r = (uint32_t)(hash2(seed ^ kWeightSalt, e) >> 32);
    return (float)(wmin + (int32_t)mulhi32(r, (uint32_t)(wmax - wmin + 1)));
}

namespace {

__global__ void k_gen_rmat(uint64_t seed, int scale, int64_t E, RmatThresholds t,
                           int32_t wmin, int32_t wmax, uint32_t *src, uint32_t *dst,
                           float *w) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t s, d;
        rmat_edge(seed, scale, (uint64_t)e, t, &s, &d);
        src[e] = s;
        dst[e] = d;
        if (w) w[e] = int_weight(seed, (uint64_t)e, wmin, wmax);
    }
}

__global__ void k_gen_uniform(uint64_t seed, uint32_t V, int64_t E, int32_t wmin,
                              int32_t wmax, uint32_t *src, uint32_t *dst, float *w) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t s, d;
        uniform_edge(seed, V, (uint64_t)e, &s, &d);
        src[e] = s;
        dst[e] = d;
        if (w) w[e] = int_weight(seed, (uint64_t)e, wmin, wmax);
    }
}

__global__ void k_check_ids(const uint32_t *src, const uint32_t *dst, int64_t E, uint32_t V,
                            int *bad) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x)
        if (src[e] >= V || dst[e] >= V) *bad = 1;
}

__global__ void k_iota(uint32_t *vals, int64_t n, int reverse) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        vals[i] = reverse ? (uint32_t)(n - 1 - i) : (uint32_t)i;
}

// keys[i] <-> keys[n-1-i]: with the edge numbers also reversed, a stable
// sort then leaves each source's edges in reverse insertion order
__global__ void k_reverse(uint32_t *keys, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n / 2;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t t = keys[i];
        keys[i] = keys[n - 1 - i];
        keys[n - 1 - i] = t;
    }
}

__global__ void k_hist(const uint32_t *keys, int64_t n, uint32_t *cnt) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[keys[i]], 1u);
}

// CSR arrays from the sorted (src, edge#) pairs.
__global__ void k_gather_csr(const uint32_t *sorted_src, const uint32_t *perm,
                             const uint32_t *dst_in, const float *w_in, int64_t E,
                             int32_t *esrc, int32_t *col, float *wt) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < E;
         k += (int64_t)gridDim.x * blockDim.x) {
        uint32_t e = perm[k];
        esrc[k] = (int32_t)sorted_src[k];
        col[k] = (int32_t)dst_in[e];
        wt[k] = w_in ? w_in[e] : 1.0f;
    }
}

// reverse-CSR arrays from the sorted (dst, csr#) pairs.
__global__ void k_gather_csc(const uint32_t *perm, const int32_t *esrc, const float *wt,
                             int64_t E, int32_t *rcol, float *rwt, int32_t *mslot) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < E;
         j += (int64_t)gridDim.x * blockDim.x) {
        uint32_t k = perm[j];
        rcol[j] = esrc[k];
        rwt[j] = wt[k];
        mslot[k] = (int32_t)j;
    }
}

__global__ void k_degrees(const int32_t *row, const int32_t *rrow, int32_t V, int32_t *outdeg,
                          int32_t *maxdeg) {
    int32_t mo = 0, mi = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V;
         v += (int64_t)gridDim.x * blockDim.x) {
        int32_t o = row[v + 1] - row[v];
        outdeg[v] = o;
        mo = max(mo, o);
        mi = max(mi, rrow[v + 1] - rrow[v]);
    }
    for (int off = 16; off; off >>= 1) {
        mo = max(mo, __shfl_xor_sync(0xffffffffu, mo, off));
        mi = max(mi, __shfl_xor_sync(0xffffffffu, mi, off));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&maxdeg[0], mo);
        atomicMax(&maxdeg[1], mi);
    }
}

int bits_for(uint32_t V) {
    int b = 0;
    while (b < 32 && (1ull << b) < (uint64_t)V) b++;
    return b;
}

}  // namespace

void graph_build_from_device_edges(Context &ctx, Graph &g, int32_t V, int64_t E,
                                   uint32_t *d_src, uint32_t *d_dst, float *d_w,
                                   uint32_t flags) {
    cudaStream_t s = ctx.stream;
    const int gridE = grid_for(E, 256, ctx.num_sms * 16);
    const int gridV = grid_for(V, 256, ctx.num_sms * 16);
    g.V = V;
    g.E = E;
    g.weighted = d_w != nullptr;
    g.device = ctx.device;
    g.row.reserve(sizeof(int32_t) * (V + 1));
    g.rrow.reserve(sizeof(int32_t) * (V + 1));
    g.outdeg.reserve(sizeof(int32_t) * (size_t)V);
    size_t eb = sizeof(int32_t) * (size_t)std::max<int64_t>(E, 1);
    g.col.reserve(eb);
    g.esrc.reserve(eb);
    g.wt.reserve(eb);
    g.rcol.reserve(eb);
    g.rwt.reserve(eb);
    g.mslot.reserve(eb);

    DevBuf cnt, vals, flag;
    try {
        flag.reserve(4 * sizeof(int));
        MB_CUDA(cudaMemsetAsync(flag.p, 0, 4 * sizeof(int), s));
        if (E > 0) {
            k_check_ids<<<gridE, 256, 0, s>>>(d_src, d_dst, E, (uint32_t)V, flag.as<int>());
            MB_CHECK_LAUNCH();
            int bad = 0;
            MB_CUDA(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            MB_CUDA(cudaStreamSynchronize(s));
            if (bad) fail(MB_ERR_INVALID, "edge endpoint outside [0, num_vertices)");
        }
        const int bits = bits_for((uint32_t)V);
        cnt.reserve(sizeof(uint32_t) * (size_t)(V + 1));
        vals.reserve(eb);

        // 1-2. CSR
        MB_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(uint32_t) * (V + 1), s));
        if (E > 0) {
            k_hist<<<gridE, 256, 0, s>>>(d_src, E, cnt.as<uint32_t>());
            MB_CHECK_LAUNCH();
        }
        scan_exclusive_u32(ctx, cnt.as<uint32_t>(), (uint32_t *)g.row.p, V + 1, nullptr, s);
        if (E > 0) {
            const int rev = (flags & MB_ORDER_REFERENCE) ? 1 : 0;
            k_iota<<<gridE, 256, 0, s>>>(vals.as<uint32_t>(), E, rev);
            if (rev) k_reverse<<<gridE, 256, 0, s>>>(d_src, E);
            MB_CHECK_LAUNCH();
            radix_sort_pairs(ctx, d_src, vals.as<uint32_t>(), E, bits, s);
            k_gather_csr<<<gridE, 256, 0, s>>>(d_src, vals.as<uint32_t>(), d_dst, d_w, E,
                                               g.esrc.as<int32_t>(), g.col.as<int32_t>(),
                                               g.wt.as<float>());
            MB_CHECK_LAUNCH();
        }
        // 3-4. reverse CSR (reuse d_dst as the key buffer, vals as the permutation)
        MB_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(uint32_t) * (V + 1), s));
        if (E > 0) {
            MB_CUDA(cudaMemcpyAsync(d_dst, g.col.p, sizeof(uint32_t) * E,
                                    cudaMemcpyDeviceToDevice, s));
            k_hist<<<gridE, 256, 0, s>>>(d_dst, E, cnt.as<uint32_t>());
            MB_CHECK_LAUNCH();
        }
        scan_exclusive_u32(ctx, cnt.as<uint32_t>(), (uint32_t *)g.rrow.p, V + 1, nullptr, s);
        if (E > 0) {
            k_iota<<<gridE, 256, 0, s>>>(vals.as<uint32_t>(), E, 0);
            MB_CHECK_LAUNCH();
            radix_sort_pairs(ctx, d_dst, vals.as<uint32_t>(), E, bits, s);
            k_gather_csc<<<gridE, 256, 0, s>>>(vals.as<uint32_t>(), g.esrc.as<int32_t>(),
                                               g.wt.as<float>(), E, g.rcol.as<int32_t>(),
                                               g.rwt.as<float>(), g.mslot.as<int32_t>());
            MB_CHECK_LAUNCH();
        }
        MB_CUDA(cudaMemsetAsync(flag.p, 0, 2 * sizeof(int), s));
        k_degrees<<<gridV, 256, 0, s>>>(g.row.as<int32_t>(), g.rrow.as<int32_t>(), V,
                                        g.outdeg.as<int32_t>(), flag.as<int32_t>());
        MB_CHECK_LAUNCH();
        int32_t md[2] = {0, 0};
        MB_CUDA(cudaMemcpyAsync(md, flag.p, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        g.max_outdeg = md[0];
        g.max_indeg = md[1];
    } catch (...) {
        cnt.release(); vals.release(); flag.release();
        throw;
    }
    cnt.release(); vals.release(); flag.release();
}

// CSR -> edge list: edge e's source is the last v with row[v] <= e (row
// checked on the host: row[0] = 0, non-decreasing, row[V] = E, so the
// search interval [0, V] always brackets e).
__global__ void k_csr_expand(const int32_t *row, int32_t V, int64_t E, uint32_t *src) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        int32_t lo = 0, hi = V;  // row[lo] <= e < row[hi]
        while (hi - lo > 1) {
            const int32_t mid = lo + ((hi - lo) >> 1);
            if ((int64_t)__ldg(&row[mid]) <= e) lo = mid; else hi = mid;
        }
        src[e] = (uint32_t)lo;
    }
}

void graph_build_from_device_csr(Context &ctx, Graph &g, int32_t V, int64_t E, const int32_t *d_row,
                                 uint32_t *d_col, float *d_w) {
    DevBuf src;
    try {
        src.reserve(sizeof(uint32_t) * (size_t)std::max<int64_t>(E, 1));
        if (E > 0) {
            k_csr_expand<<<grid_for(E, 256, ctx.num_sms * 16), 256, 0, ctx.stream>>>(d_row, V, E,
                                                                                     src.as<uint32_t>());
            MB_CHECK_LAUNCH();
        }
        // the stable sort by source keeps each row in the order given
        graph_build_from_device_edges(ctx, g, V, E, src.as<uint32_t>(), d_col, d_w, 0);
    } catch (...) {
        src.release();
        throw;
    }
    src.release();
}

// ---------------------------------------------------------------------------
// generator front ends

static void check_gen(const mb_gen_params &p) {
    if (p.wmax > 0 && (p.wmin < 0 || p.wmin > p.wmax)) fail(MB_ERR_INVALID, "bad weight range");
    switch (p.kind) {
        case MB_GEN_RMAT:
            if (p.scale < 1 || p.scale > 30) fail(MB_ERR_UNSUPPORTED, "rmat scale must be 1..30");
            if (p.num_edges < 0 || p.num_edges > 0xFFFFFFFFll)
                fail(MB_ERR_UNSUPPORTED, "num_edges must be < 2^32");
            if (p.a < 0 || p.b < 0 || p.c < 0 || p.a + p.b + p.c > 1.0 + 1e-12)
                fail(MB_ERR_INVALID, "rmat probabilities");
            break;
        case MB_GEN_UNIFORM:
            if (p.num_vertices < 1 || p.num_vertices > 0x7FFFFFFFll)
                fail(MB_ERR_UNSUPPORTED, "num_vertices must be 1..2^31-1");
            if (p.num_edges < 0 || p.num_edges > 0xFFFFFFFFll)
                fail(MB_ERR_UNSUPPORTED, "num_edges must be < 2^32");
            break;
        case MB_GEN_GRID:
            if (p.rows < 1 || p.cols < 1 || (int64_t)p.rows * p.cols > 0x7FFFFFFFll)
                fail(MB_ERR_UNSUPPORTED, "grid size");
            if (p.drop_frac < 0 || p.drop_frac > 1 || p.shortcut_frac < 0)
                fail(MB_ERR_INVALID, "grid fractions");
            break;
        default:
            fail(MB_ERR_INVALID, "unknown generator kind");
    }
}

int64_t gen_num_vertices(const mb_gen_params &p) {
    switch (p.kind) {
        case MB_GEN_RMAT: return 1ll << p.scale;
        case MB_GEN_UNIFORM: return p.num_vertices;
        default: return (int64_t)p.rows * p.cols;
    }
}

// Grid generator (host).  Undirected grid edges are numbered horizontal
// first (row-major), then vertical; each is kept with probability
// 1-drop_frac and emitted in both directions with one shared weight.  Then
// round(shortcut_frac*V) random vertex pairs are added, both directions.
static int64_t gen_grid_host(const mb_gen_params &p, int32_t *src, int32_t *dst, float *w) {
    const int64_t R = p.rows, C = p.cols, V = R * C;
    const uint64_t drop_t = (uint64_t)std::llround(p.drop_frac * 4294967296.0);
    const int64_t nh = R * (C - 1), nv = (R - 1) * C;
    int64_t m = 0;
    auto emit = [&](int64_t u, int64_t v, float wt) {
        if (src) {
            src[m] = (int32_t)u; dst[m] = (int32_t)v;
            if (w) w[m] = wt;
            src[m + 1] = (int32_t)v; dst[m + 1] = (int32_t)u;
            if (w) w[m + 1] = wt;
        }
        m += 2;
    };
    for (int64_t i = 0; i < nh + nv; i++) {
        uint64_t r = hash2(p.seed, (uint64_t)i) >> 32;
        if (r < drop_t) continue;
        int64_t u, v;
        if (i < nh) {
            int64_t rr = i / (C - 1), cc = i % (C - 1);
            u = rr * C + cc;
            v = u + 1;
        } else {
            int64_t j = i - nh;
            int64_t rr = j / C, cc = j % C;
            u = rr * C + cc;
            v = u + C;
        }
        emit(u, v, int_weight(p.seed, (uint64_t)i, p.wmin, p.wmax));
    }
    const int64_t S = std::llround(p.shortcut_frac * (double)V);
    for (int64_t k = 0; k < S; k++) {
        uint64_t h = hash2(p.seed ^ kShortcutSalt, (uint64_t)k);
        int64_t u = mulhi32((uint32_t)(h >> 32), (uint32_t)V);
        int64_t v = mulhi32((uint32_t)h, (uint32_t)V);
        emit(u, v, int_weight(p.seed ^ kShortcutSalt, (uint64_t)k, p.wmin, p.wmax));
    }
    return m;
}

int64_t generate_edges_host(const mb_gen_params &p, int32_t *src, int32_t *dst, float *w) {
    check_gen(p);
    if (p.kind == MB_GEN_GRID) return gen_grid_host(p, src, dst, w);
    const int64_t E = p.num_edges;
    if (!src) return E;
    if (p.kind == MB_GEN_RMAT) {
        RmatThresholds t = rmat_thresholds(p.a, p.b, p.c);
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < E; e++) {
            uint32_t s, d;
            rmat_edge(p.seed, p.scale, (uint64_t)e, t, &s, &d);
            src[e] = (int32_t)s;
            dst[e] = (int32_t)d;
            if (w) w[e] = int_weight(p.seed, (uint64_t)e, p.wmin, p.wmax);
        }
    } else {
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < E; e++) {
            uint32_t s, d;
            uniform_edge(p.seed, (uint32_t)p.num_vertices, (uint64_t)e, &s, &d);
            src[e] = (int32_t)s;
            dst[e] = (int32_t)d;
            if (w) w[e] = int_weight(p.seed, (uint64_t)e, p.wmin, p.wmax);
        }
    }
    return E;
}

void graph_generate(Context &ctx, Graph &g, const mb_gen_params &p, uint32_t flags) {
    check_gen(p);
    const int64_t V = gen_num_vertices(p);
    const bool weighted = p.wmax > 0;
    cudaStream_t s = ctx.stream;
    DevBuf bs, bd, bw;
    try {
        if (p.kind == MB_GEN_GRID) {
            int64_t E = gen_grid_host(p, nullptr, nullptr, nullptr);
            std::vector<int32_t> hs(E), hd(E);
            std::vector<float> hw(weighted ? E : 0);
            gen_grid_host(p, hs.data(), hd.data(), weighted ? hw.data() : nullptr);
            size_t eb = sizeof(uint32_t) * (size_t)std::max<int64_t>(E, 1);
            bs.reserve(eb);
            bd.reserve(eb);
            if (weighted) bw.reserve(eb);
            MB_CUDA(cudaMemcpyAsync(bs.p, hs.data(), 4 * E, cudaMemcpyHostToDevice, s));
            MB_CUDA(cudaMemcpyAsync(bd.p, hd.data(), 4 * E, cudaMemcpyHostToDevice, s));
            if (weighted)
                MB_CUDA(cudaMemcpyAsync(bw.p, hw.data(), 4 * E, cudaMemcpyHostToDevice, s));
            MB_CUDA(cudaStreamSynchronize(s));
            graph_build_from_device_edges(ctx, g, (int32_t)V, E, bs.as<uint32_t>(),
                                          bd.as<uint32_t>(), weighted ? bw.as<float>() : nullptr,
                                          flags);
        } else {
            const int64_t E = p.num_edges;
            size_t eb = sizeof(uint32_t) * (size_t)std::max<int64_t>(E, 1);
            bs.reserve(eb);
            bd.reserve(eb);
            if (weighted) bw.reserve(eb);
            int grid = grid_for(E, 256, ctx.num_sms * 16);
            if (E > 0) {
                if (p.kind == MB_GEN_RMAT)
                    k_gen_rmat<<<grid, 256, 0, s>>>(p.seed, p.scale, E,
                                                    rmat_thresholds(p.a, p.b, p.c), p.wmin,
                                                    p.wmax, bs.as<uint32_t>(), bd.as<uint32_t>(),
                                                    weighted ? bw.as<float>() : nullptr);
                else
                    k_gen_uniform<<<grid, 256, 0, s>>>(p.seed, (uint32_t)V, E, p.wmin, p.wmax,
                                                       bs.as<uint32_t>(), bd.as<uint32_t>(),
                                                       weighted ? bw.as<float>() : nullptr);
                MB_CHECK_LAUNCH();
            }
            graph_build_from_device_edges(ctx, g, (int32_t)V, E, bs.as<uint32_t>(),
                                          bd.as<uint32_t>(), weighted ? bw.as<float>() : nullptr,
                                          flags);
        }
    } catch (...) {
        bs.release(); bd.release(); bw.release();
        throw;
    }
    bs.release(); bd.release(); bw.release();
}

}  // namespace mb
