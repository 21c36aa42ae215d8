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
 * and that code keeps its shape here.  What changes is where application
 * data lives: the reference generates per-application SoA arrays and device
 * proxies with accessors (get_distance / set_distance, SSSP/DeviceDataStructure.h)
 * from the app's Vertex/Edge structs; here an application keeps its vertex
 * and edge attributes in medusa::DeviceArray<T> and its functors index them
 * with v.index / e.index.  The graph itself (CSR in the reference's AA edge
 * order, the reverse CSR whose positions are the message slots msgDstID) is
 * the library's (mb_graph_device_view).
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
enum FunctorType { VERTEX, EDGE, EDGELIST, MESSAGE };

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
struct Runtime {
    mb_ctx *ctx = nullptr;
    mb_graph *graph = nullptr;
    mb_graph_view view{};
    DeviceArray<MVT> msg, combined;
    DeviceArray<int> flag;
    MVT init_msg = (MVT)0;
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

/* MultipleGPU/MultiPublicAPI.h:42-100: build the graph storage from the IR. */
inline void InitHostDS(const medusa::GraphIR &ir) {
    auto &rt = MGLOBAL::rt;
    if (!rt.ctx) InitConfig("1", "0", MGLOBAL::message_mode, MGLOBAL::toExecute);
    if (rt.graph) mb_graph_destroy(rt.graph);
    rt.graph = nullptr;
    medusa::check_mb(mb_graph_from_edges(rt.ctx, ir.vertexNum, (int64_t)ir.src.size(), ir.src.data(),
                                         ir.dst.data(), ir.weight.data(), MB_ORDER_REFERENCE, &rt.graph),
                     rt.ctx, "mb_graph_from_edges");
    medusa::check_mb(mb_graph_device_view(rt.graph, &rt.view), rt.ctx, "mb_graph_device_view");
    medusa::check(cudaDeviceSynchronize(), "graph build");  // the library builds on its own stream
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
    medusa::check_mb(mb_graph_device_view(rt.graph, &rt.view), rt.ctx, "mb_graph_device_view");
    medusa::check(cudaDeviceSynchronize(), "graph build");
}

/* MultipleGPU/MultiPublicAPI.h:145-265: message buffers and the flag. */
inline void InitDeviceDS() {
    auto &rt = MGLOBAL::rt;
    int64_t n = 0;
    if (MGLOBAL::message_mode == EDGE_MESSAGE) n = rt.view.num_edges;
    else if (MGLOBAL::message_mode == VERTEX_MESSAGE) n = rt.view.num_vertices;
    rt.msg.resize(n);
    rt.combined.resize(rt.view.num_vertices);
    rt.flag.resize(1);
    MGLOBAL::super_step = 0;
    rt.sync_view();
}
inline void ResetGraphData() { MGLOBAL::super_step = 0; }

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

/* MultipleGPU/MultiPublicAPI.h:344-376: every message slot := init_val. */
template <class Message>
inline void InitMessageBuffer(const Message &init_val) {
    auto &rt = MGLOBAL::rt;
    rt.init_msg = (MVT)init_val.val;
    rt.sync_view();
    medusa::k_fill_msg<<<rt.grid(rt.msg.n), 256>>>(rt.msg.p, rt.msg.n, rt.init_msg);
    medusa::check(cudaGetLastError(), "InitMessageBuffer");
}

inline void medusa::Combiner::combineAllDevice() {
    auto &rt = MGLOBAL::rt;
    const int g = rt.grid(rt.view.num_vertices);
    switch (MGLOBAL::combiner_operator) {
        case CUDPP_ADD: k_combine<CUDPP_ADD><<<g, 256>>>(rt.combined.p); break;
        case CUDPP_MULTIPLY: k_combine<CUDPP_MULTIPLY><<<g, 256>>>(rt.combined.p); break;
        case CUDPP_MIN: k_combine<CUDPP_MIN><<<g, 256>>>(rt.combined.p); break;
        default: k_combine<CUDPP_MAX><<<g, 256>>>(rt.combined.p); break;
    }
    check(cudaGetLastError(), "combineAllDevice");
}

/* MultipleGPU/MultiAPIHoster.h:653-735 */
template <FunctorType T>
struct FunctorHolder;
template <>
struct FunctorHolder<VERTEX> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        medusa::k_vertex<<<rt.grid(rt.view.num_vertices), 256>>>(op, MGLOBAL::super_step);
        medusa::check(cudaGetLastError(), "FunctorHolder<VERTEX>");
    }
};
template <>
struct FunctorHolder<EDGE> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        medusa::k_edge<<<rt.grid(rt.view.num_edges), 256>>>(op, MGLOBAL::super_step);
        medusa::check(cudaGetLastError(), "FunctorHolder<EDGE>");
    }
};
template <>
struct FunctorHolder<EDGELIST> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        medusa::k_edgelist<<<rt.grid(rt.view.num_vertices), 256>>>(op, MGLOBAL::super_step);
        medusa::check(cudaGetLastError(), "FunctorHolder<EDGELIST>");
    }
};
template <>
struct FunctorHolder<MESSAGE> {
    template <class Op>
    static void Run(Op op) {
        auto &rt = MGLOBAL::rt;
        medusa::k_message<<<rt.grid(rt.msg.n), 256>>>(op, MGLOBAL::super_step, rt.msg.n);
        medusa::check(cudaGetLastError(), "FunctorHolder<MESSAGE>");
    }
};

/* Release the runtime's device state (the reference never frees it). */
inline void MedusaShutdown() {
    auto &rt = MGLOBAL::rt;
    rt.msg.release();
    rt.combined.release();
    rt.flag.release();
    if (rt.graph) mb_graph_destroy(rt.graph);
    rt.graph = nullptr;
    if (rt.ctx) mb_destroy(rt.ctx);
    rt.ctx = nullptr;
}

#endif /* MEDUSA_MEDUSA_H */
