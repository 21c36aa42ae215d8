// pagerank_ops.cuh -- PageRank written against the operator API, in the shape
// of the reference's MPG/UserOperators.h:16-70,175-270 and MPG/main.cu:129-169:
// every vertex sends rank/out-degree along its edge list, ADD combiner,
// rank = 0.15 + 0.85 * sum, a fixed number of supersteps.
#pragma once
#include <medusa/medusa.h>

namespace pagerank_app {

struct Message {
    MVT val;
};

// SendMsg over the edge list of a vertex (EDGELIST functor).
struct SendMsg {
    const MVT *rank;
    __device__ void operator()(D_Vertex v, EdgeList el, int super_step) {
        const int n = el.getEdgeCount();
        if (n == 0) return;
        const MVT m = rank[v.index] / (MVT)n;
        for (int k = 0; k < n; k++) el.getNextEdge().sendMsg(m);
    }
};

// UpdateVertex (MPG/UserOperators.h:16-26): "msg_sum *= 0.85" multiplies by a
// double and rounds to float, "0.15 + msg_sum" adds in double.
struct UpdateVertex {
    MVT *rank;
    __device__ void operator()(D_Vertex v, int super_step) {
        MVT sum = v.get_combined_msg();
        sum *= 0.85;
        rank[v.index] = 0.15 + sum;
    }
};

inline std::vector<MVT> run(int iters) {
    InitConfig("1", "0", EDGE_MESSAGE, false);
    MGLOBAL::combiner_datatype = CUDPP_FLOAT;
    MGLOBAL::combiner_operator = CUDPP_ADD;
    InitDeviceDS();
    const int V = MGLOBAL::rt.view.num_vertices;
    medusa::DeviceArray<MVT> rank(V);
    rank.fill((MVT)(1.0f / (float)V));
    SendMsg sm{rank.data()};
    UpdateVertex uv{rank.data()};
    Message init_msg;
    init_msg.val = 0;
    for (int it = 0; it < iters; it++) {
        InitMessageBuffer(init_msg);
        FunctorHolder<EDGELIST>::Run(sm);
        MGLOBAL::com.combineAllDevice();
        FunctorHolder<VERTEX>::Run(uv);
        MGLOBAL::super_step++;
    }
    return rank.to_host();
}

}  // namespace pagerank_app
