/* medusa/medusa.h -- Medusa's programming model (vertex / edge / edge-list /
 * message functors, message buffer, combiner, BSP loop), header-only, on top
 * of libmedusa_b200's device graph storage.
 *
 * The reference's applications (BFS, SSSP, PageRank: Algorithm/, SSSP/, MPG/)
 * are written against this model:
 *
 *   struct SendMsg { __device__ void operator()(D_Edge e, int super_step); };
 *   struct UpdateVertex { __device__ void operator()(D_Vertex v, int super_step); };
 *   void Medusa_Exec() {
 *       InitMessageBuffer(init_msg);           // MultipleGPU/MultiPublicAPI.h:344-376
 *       FunctorHolder<EDGE>::Run(send);        // MultipleGPU/MultiAPIHoster.h:653-679
 *       MGLOBAL::com.combineAllDevice();       // MedusaRT/Combiner.cu:21-142
 *       FunctorHolder<VERTEX>::Run(update);
 *   }
 *   while (exe) { ResetToExecute(); Medusa_Exec(); exe = RetriveToExecute();
 *                 MGLOBAL::super_step++; }    // SSSP/main.cu:369-382
 *
 * and that code keeps its shape here.  The reference generates, per
 * application, SoA arrays and device proxies with accessors (get_distance /
 * set_distance, SSSP/DeviceDataStructure.h:160-246) from the app's Vertex and
 * Edge structs.  Here the application lists its attributes once, before
 * including this header, and the same accessors, host arrays and device
 * arrays are generated from the list:
 *
 *   #define MEDUSA_VERTEX_FIELDS(F) F(MVT, distance) F(bool, updated)
 *   #define MEDUSA_EDGE_FIELDS(F)   // none: weight is the graph's own
 *   #include <medusa/medusa.h>
 *
 * gives D_Vertex::get_distance() / set_distance(x) / get_updated() /
 * set_updated(b), the host arrays MGLOBAL::gpu_def[0].vertexArray.distance[i]
 * (sized by InitHostDS, uploaded by InitDeviceDS) and
 * MGLOBAL::gpu_def[0].d_vertexArray.Dump(vertexArray) to read them back, as in
 * the reference's main.cu files.  The structural attributes (edge_count,
 * msg_index, edge_index, the edge's endpoints and weight) come from the
 * graph and are not listed.  An application may instead keep attributes in
 * medusa::DeviceArray<T> and index them with v.index / e.index.
 *
 * The graph itself (CSR in the reference's AA edge order, the reverse CSR
 * whose positions are the message slots msgDstID) is the library's
 * (mb_graph_device_view).
 *
 * The reference's own three apps can route their whole loop to the
 * library's hand-written kernels: one line after the functor declares that
 * the functor IS the reference's BFS, SSSP or PageRank send over the named
 * fields (MEDUSA_BUILTIN_BFS / _SSSP / _PAGERANK below), and
 * FunctorHolder<EDGE>::Run then calls mb_bfs / mb_sssp / mb_pagerank_from on
 * those fields instead of the generic functor kernels, when the fields hold
 * the state the reference's main.cu sets up (checked at the call; otherwise
 * the generic kernels run).
 *
 * Every name below is compiled into the including translation unit (nvcc,
 * -std=c++17); the functor kernels are templates instantiated for the app's
 * functors.  Built-in fast paths for the reference's own apps are the C
 * functions mb_bfs / mb_sssp / mb_pagerank of medusa_b200.h.
 */
#ifndef MEDUSA_MEDUSA_H
#define MEDUSA_MEDUSA_H

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>
#include <stdio.h>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../medusa_b200.h"

/* The message value type (the reference's Message.h: "#define MVT float"). */
#ifndef MVT
#define MVT float
#endif
#ifndef MEDUSA_MAX
#define MEDUSA_MAX 1000000000 /* SSSP/Configuration.h: unreachable distance */
#endif

/* SSSP/Configuration.h */
enum MessageMode { EDGE_MESSAGE, VERTEX_MESSAGE, NO_MESSAGE };
/* The combiner operators an app names (the reference passes CUDPP's enums,
 * SSSP/main.cu:227-228). */
enum CombinerOperator { CUDPP_ADD, CUDPP_MULTIPLY, CUDPP_MIN, CUDPP_MAX };
enum CombinerDatatype { CUDPP_INT, CUDPP_UINT, CUDPP_FLOAT };
/* MultipleGPU/MultiAPIHoster.h: the functor kinds of FunctorHolder */
enum FunctorType { VERTEX, EDGE, EDGELIST, MESSAGE, EDGE_HT };

namespace medusa {

inline void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
inline void check_mb(int rc, mb_ctx *ctx, const char *what) {
    if (rc != MB_OK) throw std::runtime_error(std::string(what) + ": " + mb_last_error(ctx));
}

/* What one functor launch reads: the graph, the message buffers, the
 * termination flag.  Copied to the translation unit's constant bank before
 * each launch (the reference keeps the same in __constant__ descriptors,
 * SSSP/DeviceDataStructure.h:7-14). */
struct RunView {
    mb_graph_view g;
    MVT *msg;       /* message slots [E] (EDGE_MESSAGE) or [V] (VERTEX_MESSAGE) */
    MVT *combined;  /* combined message per vertex [V] */
    MVT init_msg;   /* the value InitMessageBuffer filled in */
    int *to_execute;
};

}  // namespace medusa

/* One copy per translation unit (internal linkage), as the functor kernels. */
static __constant__ medusa::RunView medusa_run;

/* ---- application attributes from a field list --------------------------- */
#ifndef MEDUSA_VERTEX_FIELDS
#define MEDUSA_VERTEX_FIELDS(F)
#endif
#ifndef MEDUSA_EDGE_FIELDS
#define MEDUSA_EDGE_FIELDS(F)
#endif
#define MEDUSA_FIELD_PTR(T, name) T *name;
namespace medusa {
/* device addresses of the listed attributes (one array per field) */
struct VertexFieldPtrs {
    MEDUSA_VERTEX_FIELDS(MEDUSA_FIELD_PTR)
    char unused_;
};
struct EdgeFieldPtrs {
    MEDUSA_EDGE_FIELDS(MEDUSA_FIELD_PTR)
    char unused_;
};
}  // namespace medusa
static __constant__ medusa::VertexFieldPtrs medusa_vfields;
static __constant__ medusa::EdgeFieldPtrs medusa_efields;
#define MEDUSA_VERTEX_ACCESSORS(T, name)                                                  \
    __device__ T get_##name() const { return medusa_vfields.name[index]; }              \
    __device__ void set_##name(T value) const { medusa_vfields.name[index] = value; }
#define MEDUSA_EDGE_ACCESSORS(T, name)                                                    \
    __device__ T get_##name() const { return medusa_efields.name[index]; }              \
    __device__ void set_##name(T value) const { medusa_efields.name[index] = value; }

/* ---- device proxies ------------------------------------------------------ */

/* MedusaRT/SystemLibGPU.h */
__device__ inline void Medusa_Continue() { *medusa_run.to_execute = 1; }
__device__ inline void Medusa_Break() { *medusa_run.to_execute = 0; }

struct D_Message {
    int index;
    __device__ explicit D_Message(int i) : index(i) {}
    __device__ MVT get_val() const { return medusa_run.msg[index]; }
    __device__ void set_val(MVT v) const { medusa_run.msg[index] = v; }
};

struct D_Edge {
    int index; /* position in the CSR (the reference's edge array index) */
    __device__ explicit D_Edge(int i) : index(i) {}
    __device__ int get_srcVertexID() const { return medusa_run.g.esrc[index]; }
    __device__ int get_dstVertexID() const { return medusa_run.g.col[index]; }
    __device__ MVT get_weight() const { return medusa_run.g.wt ? (MVT)medusa_run.g.wt[index] : (MVT)1; }
    __device__ int get_msgDstID() const { return medusa_run.g.mslot[index]; }
    /* send a message along this edge: into the destination's slot msgDstID */
    __device__ void sendMsg(MVT v) const { medusa_run.msg[medusa_run.g.mslot[index]] = v; }
    MEDUSA_EDGE_FIELDS(MEDUSA_EDGE_ACCESSORS)
};

/* The out-edges of one vertex (SSSP/DeviceDataStructure.h:70-80). */
struct EdgeList {
    int start, end, cur;
    __device__ explicit EdgeList(int v)
        : start(medusa_run.g.row[v]), end(medusa_run.g.row[v + 1]), cur(medusa_run.g.row[v]) {}
    __device__ int getEdgeCount() const { return end - start; }
    __device__ D_Edge getNextEdge() { return D_Edge(cur++); }
    __device__ D_Edge getPreviousEdge() { return D_Edge(--cur); }
    __device__ D_Edge operator[](int k) const { return D_Edge(start + k); }
};

struct D_Vertex {
    int index;
    __device__ explicit D_Vertex(int i) : index(i) {}
    __device__ int get_edge_count() const { return medusa_run.g.outdeg[index]; }
    __device__ int get_msg_index() const { return medusa_run.g.rrow[index]; }
    __device__ int get_msg_count() const { return medusa_run.g.rrow[index + 1] - medusa_run.g.rrow[index]; }
    /* the combiner's result for this vertex (SSSP/DeviceDataStructure.h:221-235);
     * a vertex without messages gets the buffer's initial value */
    __device__ MVT get_combined_msg() const { return medusa_run.combined[index]; }
    MEDUSA_VERTEX_FIELDS(MEDUSA_VERTEX_ACCESSORS)
};

namespace medusa {

/* ---- functor kernels -------------------------------------------------------- */

template <class Op>
__global__ void k_vertex(Op op, int super_step) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < medusa_run.g.num_vertices;
         v += (int64_t)gridDim.x * blockDim.x)
        op(D_Vertex((int)v), super_step);
}
template <class Op>
__global__ void k_edge(Op op, int super_step) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < medusa_run.g.num_edges;
         e += (int64_t)gridDim.x * blockDim.x)
        op(D_Edge((int)e), super_step);
}
template <class Op>
__global__ void k_edgelist(Op op, int super_step) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < medusa_run.g.num_vertices;
         v += (int64_t)gridDim.x * blockDim.x)
        op(D_Vertex((int)v), EdgeList((int)v), super_step);
}
template <class Op>
__global__ void k_message(Op op, int super_step, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        op(D_Message((int)i), super_step);
}
static __global__ void k_fill_msg(MVT *m, int64_t n, MVT v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m[i] = v;
}
/* Combine the messages of each vertex, slots rrow[v] .. rrow[v+1]-1, folded in
 * slot order -- the order of the reference's CPU combine
 * (MPG/CPUFunctorHoster.cpp:21-26, SSSP/CPUFunctorHoster.cpp:17-22). */
template <int kOp>
__global__ void k_combine(MVT *combined) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < medusa_run.g.num_vertices;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int b = medusa_run.g.rrow[v], e = medusa_run.g.rrow[v + 1];
        MVT acc;
        if (b == e) {
            acc = medusa_run.init_msg;
        } else if (kOp == CUDPP_ADD) {
            acc = (MVT)0;
            for (int j = b; j < e; j++) acc += medusa_run.msg[j];
        } else if (kOp == CUDPP_MULTIPLY) {
            acc = (MVT)1;
            for (int j = b; j < e; j++) acc *= medusa_run.msg[j];
        } else {
            acc = medusa_run.msg[b];
            for (int j = b + 1; j < e; j++) {
                const MVT m = medusa_run.msg[j];
                acc = (kOp == CUDPP_MIN) ? (m < acc ? m : acc) : (m > acc ? m : acc);
            }
        }
        combined[v] = acc;
    }
}

/* Device array of an application attribute (vertex or edge field). */
template <class T>
struct DeviceArray {
    T *p = nullptr;
    int64_t n = 0;
    DeviceArray() = default;
    explicit DeviceArray(int64_t count) { resize(count); }
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    DeviceArray(DeviceArray &&o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DeviceArray &operator=(DeviceArray &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DeviceArray() { release(); }
    void resize(int64_t count) {
        release();
        n = count;
        check(cudaMalloc(&p, sizeof(T) * (size_t)(count > 0 ? count : 1)), "cudaMalloc");
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void upload(const T *host) { check(cudaMemcpy(p, host, sizeof(T) * (size_t)n, cudaMemcpyHostToDevice), "upload"); }
    void download(T *host) const { check(cudaMemcpy(host, p, sizeof(T) * (size_t)n, cudaMemcpyDeviceToHost), "download"); }
    std::vector<T> to_host() const {
        std::vector<T> h((size_t)n);
        if (n) download(h.data());
        return h;
    }
    void fill(const T &v) {
        std::vector<T> h((size_t)n, v);
        if (n) upload(h.data());
    }
    T *data() const { return p; }
};

/* Host array of one attribute (bool-safe, unlike std::vector<bool>). */
template <class T>
struct HostArray {
    std::unique_ptr<T[]> p;
    int64_t n = 0;
    void resize(int64_t count) {
        p.reset(new T[(size_t)(count > 0 ? count : 1)]());
        n = count;
    }
    T &operator[](int64_t i) { return p[(size_t)i]; }
    const T &operator[](int64_t i) const { return p[(size_t)i]; }
    T *data() const { return p.get(); }
};

/* The listed attributes as host arrays (the reference's VertexArray /
 * EdgeArray, SSSP/VertexDataType.h, SSSP/EdgeDataType.h) and device arrays
 * (D_VertexArray / D_EdgeArray, with Fill and Dump). */
#define MEDUSA_HOST_FIELD(T, name) HostArray<T> name;
#define MEDUSA_DEV_FIELD(T, name) DeviceArray<T> name;
#define MEDUSA_RESIZE_FIELD(T, name) name.resize(count);
#define MEDUSA_FILL_FIELD(T, name) \
    name.resize(h.size);           \
    if (h.size) name.upload(h.name.data());
#define MEDUSA_DUMP_FIELD(T, name) \
    if (size) name.download(h.name.data());
#define MEDUSA_PTR_FIELD(T, name) out.name = name.p;
struct VertexArray {
    int size = 0;
    MEDUSA_VERTEX_FIELDS(MEDUSA_HOST_FIELD)
    void resize(int count) {
        size = count;
        MEDUSA_VERTEX_FIELDS(MEDUSA_RESIZE_FIELD)
    }
};
struct D_VertexArray {
    int size = 0;
    MEDUSA_VERTEX_FIELDS(MEDUSA_DEV_FIELD)
    void Fill(const VertexArray &h) {
        size = h.size;
        MEDUSA_VERTEX_FIELDS(MEDUSA_FILL_FIELD)
    }
    void Dump(VertexArray &h) const {
        if (h.size != size) h.resize(size);
        MEDUSA_VERTEX_FIELDS(MEDUSA_DUMP_FIELD)
    }
    VertexFieldPtrs ptrs() const {
        VertexFieldPtrs out{};
        MEDUSA_VERTEX_FIELDS(MEDUSA_PTR_FIELD)
        return out;
    }
};
struct EdgeArray {
    int size = 0;
    MEDUSA_EDGE_FIELDS(MEDUSA_HOST_FIELD)
    void resize(int count) {
        size = count;
        MEDUSA_EDGE_FIELDS(MEDUSA_RESIZE_FIELD)
    }
};
struct D_EdgeArray {
    int size = 0;
    MEDUSA_EDGE_FIELDS(MEDUSA_DEV_FIELD)
    void Fill(const EdgeArray &h) {
        size = h.size;
        MEDUSA_EDGE_FIELDS(MEDUSA_FILL_FIELD)
    }
    void Dump(EdgeArray &h) const {
        if (h.size != size) h.resize(size);
        MEDUSA_EDGE_FIELDS(MEDUSA_DUMP_FIELD)
    }
    EdgeFieldPtrs ptrs() const {
        EdgeFieldPtrs out{};
        MEDUSA_EDGE_FIELDS(MEDUSA_PTR_FIELD)
        return out;
    }
};
/* One GPU's share of the application data (MultipleGPU/MultiGraphStorage.h's
 * gpu_def[i]; one GPU here).  Edge attributes are indexed by the edge's
 * position in the AA order (D_Edge::index). */
struct GPUDef {
    VertexArray vertexArray;
    D_VertexArray d_vertexArray;
    EdgeArray edgeArray;
    D_EdgeArray d_edgeArray;
};

/* ---- graph construction ------------------------------------------------------ */

/* The edge an application adds (SSSP/Edge.h: srcVertexID, dstVertexID, weight). */
struct Edge {
    int srcVertexID;
    int dstVertexID;
    float weight;
};

/* MedusaRT/GraphConverter.h GraphIR: vertices 0..n-1, edges added one by
 * one; the device graph keeps the reference's AA order (each vertex's edges
 * in reverse insertion order, as AddEdge prepends). */
struct GraphIR {
    int vertexNum = 0;
    int totalEdgeCount = 0;
    std::vector<int32_t> src, dst;
    std::vector<float> weight;
    GraphIR() = default;
    explicit GraphIR(int num) { resize(num); }
    void resize(int num) {
        vertexNum = num;
        totalEdgeCount = 0;
        src.clear();
        dst.clear();
        weight.clear();
    }
    void AddEdge(Edge e) {
        src.push_back(e.srcVertexID);
        dst.push_back(e.dstVertexID);
        weight.push_back(e.weight);
        totalEdgeCount++;
    }
};

}  // namespace medusa

/* ---- the runtime (MGLOBAL, MultipleGPU/MultiGraphStorage.cu:11-29) ----------- */

namespace medusa {
struct Combiner {
    void combineAllDevice();
};
/* Which built-in path ran the last superstep (MEDUSA_BUILTIN_*), with the
 * library's statistics of that call. */
enum BuiltinApp { BUILTIN_NONE = 0, BUILTIN_BFS = 1, BUILTIN_SSSP = 2, BUILTIN_PAGERANK = 3 };
struct Runtime {
    mb_ctx *ctx = nullptr;
    mb_graph *graph = nullptr;
    mb_graph_view view{};
    DeviceArray<MVT> msg, combined;
    DeviceArray<int> flag;
    MVT init_msg = (MVT)0;
    bool fill_pending = false;      /* InitMessageBuffer ran; the fill waits for a reader */
    int skip_step = -1;             /* a built-in path finished this superstep */
    bool builtin_enabled = true;    /* route MEDUSA_BUILTIN_* functors to the library */
    int64_t generic_launches = 0;   /* functor / combiner kernels launched */
    BuiltinApp last_builtin = BUILTIN_NONE;
    mb_stats builtin_stats{};
    int num_sms = 148;
    cudaStream_t stream = 0;
    void sync_view() {
        RunView rv;
        rv.g = view;
        rv.msg = msg.p;
        rv.combined = combined.p;
        rv.init_msg = init_msg;
        rv.to_execute = flag.p;
        check(cudaMemcpyToSymbol(medusa_run, &rv, sizeof(rv)), "constant");
    }
    int grid(int64_t n) const {
        int64_t b = (n + 255) / 256;
        if (b < 1) b = 1;
        if (b > (int64_t)num_sms * 8) b = (int64_t)num_sms * 8;
        return (int)b;
    }
    void fill_messages();
};
}  // namespace medusa

namespace MGLOBAL {
inline int super_step = 0;
inline int num_gpu_to_use = 1;
inline MessageMode message_mode = EDGE_MESSAGE;
inline CombinerOperator combiner_operator = CUDPP_ADD;
inline CombinerDatatype combiner_datatype = CUDPP_FLOAT;
inline bool toExecute = false;
inline medusa::Combiner com;
inline medusa::Runtime rt;
inline medusa::GPUDef gpu_def[1];
}  // namespace MGLOBAL

/* MultipleGPU/MultiPublicAPI.h:15-35.  gpu_num must be "1" (one GPU). */
inline void InitConfig(const char *gpu_num, const char *max_hop, MessageMode mm, bool exe) {
    (void)max_hop; /* multi-hop replicas: MultipleGPU only */
    if (gpu_num && atoi(gpu_num) != 1) throw std::runtime_error("this build runs on one GPU");
    MGLOBAL::num_gpu_to_use = 1;
    MGLOBAL::message_mode = mm;
    MGLOBAL::toExecute = exe;
    MGLOBAL::super_step = 0;
    if (!MGLOBAL::rt.ctx) medusa::check_mb(mb_create(0, &MGLOBAL::rt.ctx), nullptr, "mb_create");
    cudaDeviceProp prop;
    medusa::check(cudaGetDeviceProperties(&prop, 0), "device properties");
    MGLOBAL::rt.num_sms = prop.multiProcessorCount;
}

namespace medusa {
/* After the graph is built: the application's host arrays are sized to it. */
inline void graph_ready() {
    auto &rt = MGLOBAL::rt;
    medusa::check_mb(mb_graph_device_view(rt.graph, &rt.view), rt.ctx, "mb_graph_device_view");
    medusa::check(cudaDeviceSynchronize(), "graph build");  // the library builds on its own stream
    MGLOBAL::gpu_def[0].vertexArray.resize(rt.view.num_vertices);
    MGLOBAL::gpu_def[0].edgeArray.resize((int)rt.view.num_edges);
}
}  // namespace medusa

/* MultipleGPU/MultiPublicAPI.h:42-100: build the graph storage from the IR. */
inline void InitHostDS(const medusa::GraphIR &ir) {
    auto &rt = MGLOBAL::rt;
    if (!rt.ctx) InitConfig("1", "0", MGLOBAL::message_mode, MGLOBAL::toExecute);
    if (rt.graph) mb_graph_destroy(rt.graph);
    rt.graph = nullptr;
    medusa::check_mb(mb_graph_from_edges(rt.ctx, ir.vertexNum, (int64_t)ir.src.size(), ir.src.data(),
                                         ir.dst.data(), ir.weight.data(), MB_ORDER_REFERENCE, &rt.graph),
                     rt.ctx, "mb_graph_from_edges");
    medusa::graph_ready();
}

/* The same from GTgraph text (parsed on the GPU), the reference's file format. */
inline void InitHostDSFromGTGraph(const std::string &path) {
    auto &rt = MGLOBAL::rt;
    if (!rt.ctx) InitConfig("1", "0", MGLOBAL::message_mode, MGLOBAL::toExecute);
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    if (rt.graph) mb_graph_destroy(rt.graph);
    rt.graph = nullptr;
    medusa::check_mb(mb_graph_from_gtgraph(rt.ctx, text.data(), (int64_t)text.size(), MB_ORDER_REFERENCE,
                                           &rt.graph),
                     rt.ctx, "mb_graph_from_gtgraph");
    medusa::graph_ready();
}

namespace medusa {
/* The application's attributes to the device, and their addresses to the
 * functors' constant bank. */
inline void upload_fields() {
    auto &d = MGLOBAL::gpu_def[0];
    d.d_vertexArray.Fill(d.vertexArray);
    d.d_edgeArray.Fill(d.edgeArray);
    const VertexFieldPtrs vp = d.d_vertexArray.ptrs();
    const EdgeFieldPtrs ep = d.d_edgeArray.ptrs();
    check(cudaMemcpyToSymbol(medusa_vfields, &vp, sizeof(vp)), "vertex fields");
    check(cudaMemcpyToSymbol(medusa_efields, &ep, sizeof(ep)), "edge fields");
}
}  // namespace medusa

/* MultipleGPU/MultiPublicAPI.h:145-265: message buffers, the flag, and the
 * application's attributes (the reference's D_VertexArray::Fill). */
inline void InitDeviceDS() {
    auto &rt = MGLOBAL::rt;
    int64_t n = 0;
    if (MGLOBAL::message_mode == EDGE_MESSAGE) n = rt.view.num_edges;
    else if (MGLOBAL::message_mode == VERTEX_MESSAGE) n = rt.view.num_vertices;
    rt.msg.resize(n);
    rt.combined.resize(rt.view.num_vertices);
    rt.flag.resize(1);
    rt.fill_pending = false;
    rt.skip_step = -1;
    MGLOBAL::super_step = 0;
    rt.sync_view();
    medusa::upload_fields();
    int v = MGLOBAL::toExecute ? 1 : 0;  // the flag starts as InitConfig's exe
    medusa::check(cudaMemcpy(rt.flag.p, &v, sizeof(int), cudaMemcpyHostToDevice), "InitDeviceDS");
}
/* Back to the state the host arrays hold, for another run. */
inline void ResetGraphData() {
    MGLOBAL::super_step = 0;
    MGLOBAL::rt.skip_step = -1;
    medusa::upload_fields();
}

/* MultipleGPU/MultiUtilities.h:48-69 */
inline void ResetToExecute() {
    int v = MGLOBAL::toExecute ? 1 : 0;
    medusa::check(cudaMemcpy(MGLOBAL::rt.flag.p, &v, sizeof(int), cudaMemcpyHostToDevice), "ResetToExecute");
}
inline bool RetriveToExecute() {
    int v = 0;
    medusa::check(cudaMemcpy(&v, MGLOBAL::rt.flag.p, sizeof(int), cudaMemcpyDeviceToHost), "RetriveToExecute");
    return v != 0;
}

namespace medusa {
inline bool skipping() { return MGLOBAL::rt.skip_step == MGLOBAL::super_step; }
inline void Runtime::fill_messages() {
    if (!fill_pending) return;
    fill_pending = false;
    k_fill_msg<<<grid(msg.n), 256>>>(msg.p, msg.n, init_msg);
    generic_launches++;
    check(cudaGetLastError(), "InitMessageBuffer");
}
}  // namespace medusa

/* MultipleGPU/MultiPublicAPI.h:344-376: every message slot := init_val.  The
 * fill itself runs when a functor or the combiner first reads the buffer (a
 * superstep that a built-in path runs whole never needs it). */
template <class Message>
inline void InitMessageBuffer(const Message &init_val) {
    auto &rt = MGLOBAL::rt;
    if (medusa::skipping()) return;
    rt.init_msg = (MVT)init_val.val;
    rt.sync_view();
    rt.fill_pending = true;
}

inline void medusa::Combiner::combineAllDevice() {
    auto &rt = MGLOBAL::rt;
    if (skipping()) return;
    rt.fill_messages();
    const int g = rt.grid(rt.view.num_vertices);
    switch (MGLOBAL::combiner_operator) {
        case CUDPP_ADD: k_combine<CUDPP_ADD><<<g, 256>>>(rt.combined.p); break;
        case CUDPP_MULTIPLY: k_combine<CUDPP_MULTIPLY><<<g, 256>>>(rt.combined.p); break;
        case CUDPP_MIN: k_combine<CUDPP_MIN><<<g, 256>>>(rt.combined.p); break;
        default: k_combine<CUDPP_MAX><<<g, 256>>>(rt.combined.p); break;
    }
    rt.generic_launches++;
    check(cudaGetLastError(), "combineAllDevice");
}

/* ---- the reference's three apps on the library's kernels ------------------- */
/* An application declares, after its edge functor, that the functor is the
 * reference's BFS, SSSP or PageRank send over the named vertex fields:
 *
 *   MEDUSA_BUILTIN_BFS(UpdateLevel, level)            Algorithm/UserOperators.h:17-35
 *   MEDUSA_BUILTIN_SSSP(SendMsg, distance, updated)   SSSP/UserOperators.h:151-189
 *   MEDUSA_BUILTIN_PAGERANK(SendMsg, level)           MPG/UserOperators.h:16-43
 *
 * FunctorHolder<EDGE>::Run(op) then hands the superstep to the library:
 *   BFS: at superstep 0, with level 0 at the roots and MVT_Init_Value (-1)
 *     elsewhere, the whole traversal runs in mb_bfs (levels of several roots
 *     are combined by minimum) and the loop's flag is left clear;
 *   SSSP: at superstep 0, with updated set exactly on the vertices at
 *     distance 0 and MEDUSA_MAX elsewhere, the whole traversal runs in
 *     mb_sssp, every vertex ends not updated, and the flag is left clear;
 *   PageRank: each superstep is mb_pagerank_from(1 superstep) from the rank
 *     field into the rank field (send rank/edge_count, sum, 0.15 + 0.85 sum).
 * The rest of that superstep's Medusa_Exec (InitMessageBuffer, the combiner,
 * the vertex functor) then does nothing.  When the fields hold anything else
 * the generic functor kernels run as usual.  MGLOBAL::rt.last_builtin and
 * builtin_stats say what ran (kernel launches, schedules per superstep). */
namespace medusa {
template <class Op>
struct Builtin {
    static constexpr BuiltinApp app = BUILTIN_NONE;
    static int *level() { return nullptr; }
    static float *dist() { return nullptr; }
    static bool *updated() { return nullptr; }
    static float *rank() { return nullptr; }
};

static __global__ void k_min_levels(const int32_t *lv, int32_t nsrc, int64_t V, int *out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
        int best = -1;
        for (int32_t s = 0; s < nsrc; s++) {
            const int x = lv[s * V + v];
            if (x >= 0 && (best < 0 || x < best)) best = x;
        }
        out[v] = best;
    }
}
static __global__ void k_min_dist(const float *d, int32_t nsrc, int64_t V, float *out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
        float best = d[v];
        for (int32_t s = 1; s < nsrc; s++) best = fminf(best, d[s * V + v]);
        out[v] = best;
    }
}

/* Levels (or distances) of several roots, combined by minimum. */
inline bool builtin_bfs(int *level) {
    auto &rt = MGLOBAL::rt;
    const int64_t V = rt.view.num_vertices;
    if (MGLOBAL::super_step != 0 || !level) return false;
    std::vector<int> h((size_t)V);
    if (V) check(cudaMemcpy(h.data(), level, sizeof(int) * (size_t)V, cudaMemcpyDeviceToHost), "BFS roots");
    std::vector<int32_t> roots;
    for (int64_t v = 0; v < V; v++) {
        if (h[v] == 0) roots.push_back((int32_t)v);
        else if (h[v] != -1) return false;
    }
    if (roots.empty()) return false;
    if (roots.size() == 1) {
        check_mb(mb_bfs(rt.ctx, rt.graph, roots.data(), 1, level, &rt.builtin_stats), rt.ctx, "mb_bfs");
    } else {
        DeviceArray<int32_t> all((int64_t)roots.size() * V);
        check_mb(mb_bfs(rt.ctx, rt.graph, roots.data(), (int32_t)roots.size(), all.p, &rt.builtin_stats),
                 rt.ctx, "mb_bfs");
        k_min_levels<<<rt.grid(V), 256>>>(all.p, (int32_t)roots.size(), V, level);
        check(cudaDeviceSynchronize(), "BFS roots combined");
    }
    return true;
}

inline bool builtin_sssp(float *dist, bool *updated) {
    auto &rt = MGLOBAL::rt;
    const int64_t V = rt.view.num_vertices;
    if (MGLOBAL::super_step != 0 || !dist || !updated) return false;
    std::vector<float> hd((size_t)V);
    std::unique_ptr<bool[]> hu(new bool[(size_t)(V > 0 ? V : 1)]);
    if (V) {
        check(cudaMemcpy(hd.data(), dist, sizeof(float) * (size_t)V, cudaMemcpyDeviceToHost), "SSSP state");
        check(cudaMemcpy(hu.get(), updated, sizeof(bool) * (size_t)V, cudaMemcpyDeviceToHost), "SSSP state");
    }
    std::vector<int32_t> roots;
    for (int64_t v = 0; v < V; v++) {
        if (hu[v] && hd[v] == 0.0f) roots.push_back((int32_t)v);
        else if (hu[v] || hd[v] != (float)MEDUSA_MAX) return false;
    }
    if (roots.empty()) return false;
    if (roots.size() == 1) {
        check_mb(mb_sssp(rt.ctx, rt.graph, roots.data(), 1, dist, &rt.builtin_stats), rt.ctx, "mb_sssp");
    } else {
        DeviceArray<float> all((int64_t)roots.size() * V);
        check_mb(mb_sssp(rt.ctx, rt.graph, roots.data(), (int32_t)roots.size(), all.p, &rt.builtin_stats),
                 rt.ctx, "mb_sssp");
        k_min_dist<<<rt.grid(V), 256>>>(all.p, (int32_t)roots.size(), V, dist);
    }
    check(cudaMemset(updated, 0, sizeof(bool) * (size_t)V), "SSSP updated");
    check(cudaDeviceSynchronize(), "SSSP");
    return true;
}

inline bool builtin_pagerank(float *rank) {
    auto &rt = MGLOBAL::rt;
    if (!rank || MGLOBAL::combiner_operator != CUDPP_ADD) return false;
    check_mb(mb_pagerank_from(rt.ctx, rt.graph, 1, rank, rank, &rt.builtin_stats), rt.ctx, "mb_pagerank_from");
    return true;
}

template <class Op>
inline bool run_builtin() {
    auto &rt = MGLOBAL::rt;
    using B = Builtin<Op>;
    bool ran = false;
    if (B::app == BUILTIN_BFS) ran = builtin_bfs(B::level());
    else if (B::app == BUILTIN_SSSP) ran = builtin_sssp(B::dist(), B::updated());
    else if (B::app == BUILTIN_PAGERANK) ran = builtin_pagerank(B::rank());
    if (!ran) return false;
    if (B::app != BUILTIN_PAGERANK) {  // the traversal is complete: no further superstep
        const int zero = 0;
        check(cudaMemcpy(rt.flag.p, &zero, sizeof(int), cudaMemcpyHostToDevice), "flag");
    }
    rt.fill_pending = false;
    rt.skip_step = MGLOBAL::super_step;
    rt.last_builtin = B::app;
    return true;
}
}  // namespace medusa

#define MEDUSA_BUILTIN_BFS(Functor, level_field)                                                   \
    template <>                                                                                     \
    struct medusa::Builtin<Functor> {                                                               \
        static constexpr medusa::BuiltinApp app = medusa::BUILTIN_BFS;                              \
        static int *level() { return (int *)MGLOBAL::gpu_def[0].d_vertexArray.level_field.p; }      \
        static float *dist() { return nullptr; }                                                    \
        static bool *updated() { return nullptr; }                                                  \
        static float *rank() { return nullptr; }                                                    \
    };
#define MEDUSA_BUILTIN_SSSP(Functor, dist_field, updated_field)                                    \
    template <>                                                                                     \
    struct medusa::Builtin<Functor> {                                                               \
        static constexpr medusa::BuiltinApp app = medusa::BUILTIN_SSSP;                             \
        static int *level() { return nullptr; }                                                     \
        static float *dist() { return (float *)MGLOBAL::gpu_def[0].d_vertexArray.dist_field.p; }    \
        static bool *updated() { return (bool *)MGLOBAL::gpu_def[0].d_vertexArray.updated_field.p; } \
        static float *rank() { return nullptr; }                                                    \
    };
#define MEDUSA_BUILTIN_PAGERANK(Functor, rank_field)                                               \
    template <>                                                                                     \
    struct medusa::Builtin<Functor> {                                                               \
        static constexpr medusa::BuiltinApp app = medusa::BUILTIN_PAGERANK;                         \
        static int *level() { return nullptr; }                                                     \
        static float *dist() { return nullptr; }                                                    \
        static bool *updated() { return nullptr; }                                                  \
        static float *rank() { return (float *)MGLOBAL::gpu_def[0].d_vertexArray.rank_field.p; }    \
    };

/* MultipleGPU/MultiAPIHoster.h:653-735 */
template <FunctorType T>
struct FunctorHolder;
template <>
struct FunctorHolder<VERTEX> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        if (medusa::skipping()) return;
        medusa::k_vertex<<<rt.grid(rt.view.num_vertices), 256>>>(op, MGLOBAL::super_step);
        rt.generic_launches++;
        medusa::check(cudaGetLastError(), "FunctorHolder<VERTEX>");
    }
};
template <>
struct FunctorHolder<EDGE> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        if (medusa::skipping()) return;
        if (medusa::Builtin<Op>::app != medusa::BUILTIN_NONE && rt.builtin_enabled && medusa::run_builtin<Op>())
            return;
        rt.fill_messages();
        medusa::k_edge<<<rt.grid(rt.view.num_edges), 256>>>(op, MGLOBAL::super_step);
        rt.generic_launches++;
        medusa::check(cudaGetLastError(), "FunctorHolder<EDGE>");
    }
};
/* The edge functor on a fixed small grid, one CTA per SM, each thread
 * walking many edges (the reference's hash-table variant, 60 x 256 threads,
 * MultipleGPU/MultiAPIHoster.h:682-703, MedusaRT/APIKernelWrappers.h:185-193). */
template <>
struct FunctorHolder<EDGE_HT> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        if (medusa::skipping()) return;
        rt.fill_messages();
        medusa::k_edge<<<rt.num_sms, 256>>>(op, MGLOBAL::super_step);
        rt.generic_launches++;
        medusa::check(cudaGetLastError(), "FunctorHolder<EDGE_HT>");
    }
};
template <>
struct FunctorHolder<EDGELIST> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        if (medusa::skipping()) return;
        rt.fill_messages();
        medusa::k_edgelist<<<rt.grid(rt.view.num_vertices), 256>>>(op, MGLOBAL::super_step);
        rt.generic_launches++;
        medusa::check(cudaGetLastError(), "FunctorHolder<EDGELIST>");
    }
};
template <>
struct FunctorHolder<MESSAGE> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        if (medusa::skipping()) return;
        rt.fill_messages();
        medusa::k_message<<<rt.grid(rt.msg.n), 256>>>(op, MGLOBAL::super_step, rt.msg.n);
        rt.generic_launches++;
        medusa::check(cudaGetLastError(), "FunctorHolder<MESSAGE>");
    }
};

/* Release the runtime's device state (the reference never frees it). */
inline void MedusaShutdown() {
    auto &rt = MGLOBAL::rt;
    rt.msg.release();
    rt.combined.release();
    rt.flag.release();
    MGLOBAL::gpu_def[0].d_vertexArray = medusa::D_VertexArray{};
    MGLOBAL::gpu_def[0].d_edgeArray = medusa::D_EdgeArray{};
    if (rt.graph) mb_graph_destroy(rt.graph);
    rt.graph = nullptr;
    if (rt.ctx) mb_destroy(rt.ctx);
    rt.ctx = nullptr;
}

#endif /* MEDUSA_MEDUSA_H */
