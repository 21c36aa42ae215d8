// msg_ops.cuh -- the two remaining functor kinds of the operator API:
// FunctorHolder<EDGE_HT> (the edge functor on a small fixed grid, the
// reference's hash-table variant, MultipleGPU/MultiAPIHoster.h:682-703) and
// FunctorHolder<MESSAGE> (a functor over every message slot between the send
// and the combiner, MultipleGPU/MultiAPIHoster.h:720-735,
// MedusaRT/APIKernelWrappers.h:209-218).
//
// The app is PageRank with the damping moved onto the messages: the send
// (EDGE_HT) writes rank/out-degree into each slot, a MESSAGE functor scales
// every message by 0.85 (float times a double constant, rounded to float),
// the ADD combiner folds each vertex's slots in slot order, and the update
// sets rank = 0.15 + sum (a double add rounded to float).
#pragma once
#include <medusa/medusa.h>

namespace msg_app {

struct Message {
    MVT val;
};

struct SendMsg {
    const MVT *rank;
    const int *outdeg;
    __device__ void operator()(D_Edge e, int super_step) {
        const int u = e.get_srcVertexID();
        e.sendMsg(rank[u] / (MVT)outdeg[u]);
    }
};

struct DampMsg {
    __device__ void operator()(D_Message m, int super_step) {
        MVT x = m.get_val();
        x *= 0.85;
        m.set_val(x);
    }
};

struct UpdateVertex {
    MVT *rank;
    __device__ void operator()(D_Vertex v, int super_step) { rank[v.index] = 0.15 + v.get_combined_msg(); }
};

inline std::vector<MVT> run(int iters) {
    InitConfig("1", "0", EDGE_MESSAGE, false);
    MGLOBAL::combiner_datatype = CUDPP_FLOAT;
    MGLOBAL::combiner_operator = CUDPP_ADD;
    InitDeviceDS();
    const int V = MGLOBAL::rt.view.num_vertices;
    medusa::DeviceArray<MVT> rank(V);
    rank.fill((MVT)(1.0f / (float)V));
    SendMsg sm{rank.data(), MGLOBAL::rt.view.outdeg};
    DampMsg dm;
    UpdateVertex uv{rank.data()};
    Message init_msg;
    init_msg.val = 0;
    for (int it = 0; it < iters; it++) {
        InitMessageBuffer(init_msg);
        FunctorHolder<EDGE_HT>::Run(sm);
        FunctorHolder<MESSAGE>::Run(dm);
        MGLOBAL::com.combineAllDevice();
        FunctorHolder<VERTEX>::Run(uv);
        MGLOBAL::super_step++;
    }
    return rank.to_host();
}

}  // namespace msg_app
