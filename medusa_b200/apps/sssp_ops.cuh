// sssp_ops.cuh -- SSSP written against the operator API, in the shape of the
// reference's SSSP/UserOperators.h:151-264 and SSSP/main.cu:227-382: send
// along the edges of updated vertices, MIN combiner, update.
#pragma once
#include <medusa/medusa.h>

namespace sssp_app {

struct Message {
    MVT val;
};

// SendMsg: an updated source offers its distance plus the edge weight.
struct SendMsg {
    const MVT *distance;
    const int *updated;
    __device__ void operator()(D_Edge e, int super_step) {
        const int src = e.get_srcVertexID();
        if (updated[src]) e.sendMsg(distance[src] + e.get_weight());
    }
};

// UpdateVertex: take the combined minimum if it is shorter.
struct UpdateVertex {
    MVT *distance;
    int *updated;
    __device__ void operator()(D_Vertex v, int super_step) {
        const MVT m = v.get_combined_msg();
        if (m < distance[v.index]) {
            distance[v.index] = m;
            updated[v.index] = 1;
            Medusa_Continue();
        } else {
            updated[v.index] = 0;
        }
    }
};

inline std::vector<MVT> run(int source) {
    InitConfig("1", "0", EDGE_MESSAGE, false);
    MGLOBAL::combiner_datatype = CUDPP_FLOAT;
    MGLOBAL::combiner_operator = CUDPP_MIN;
    InitDeviceDS();
    const int V = MGLOBAL::rt.view.num_vertices;
    medusa::DeviceArray<MVT> distance(V);
    medusa::DeviceArray<int> updated(V);
    std::vector<MVT> hd(V, (MVT)MEDUSA_MAX);
    std::vector<int> hu(V, 0);
    hd[source] = 0;
    hu[source] = 1;
    distance.upload(hd.data());
    updated.upload(hu.data());
    SendMsg sm{distance.data(), updated.data()};
    UpdateVertex uv{distance.data(), updated.data()};
    Message init_msg;
    init_msg.val = FLT_MAX;
    bool exe = true;
    while (exe) {
        ResetToExecute();
        InitMessageBuffer(init_msg);
        FunctorHolder<EDGE>::Run(sm);
        MGLOBAL::com.combineAllDevice();
        FunctorHolder<VERTEX>::Run(uv);
        exe = RetriveToExecute();
        MGLOBAL::super_step++;
    }
    return distance.to_host();
}

}  // namespace sssp_app
