// dropin_sssp.cu -- the reference's SSSP app (SSSP/Vertex.h,
// SSSP/UserOperators.h:151-264, SSSP/main.cu:300-382) as it compiles against
// include/medusa/medusa.h: the Vertex struct's attributes become a field
// list, the functors and the BSP loop keep their shape, and one line routes
// the send functor to the library's SSSP (mb_sssp).  The functor bodies are
// the reference's algorithm written against the same accessor API.
#define MEDUSA_VERTEX_FIELDS(F) F(MVT, distance) F(bool, updated)
#include <medusa/medusa.h>

#include "dropin_common.h"

struct Message {
    MVT val;
};

// a vertex whose combined message beats its distance takes it and stays active
struct UpdateVertex {
    __device__ void operator()(D_Vertex vertex, int super_step) {
        const MVT best = vertex.get_combined_msg();
        if (best < vertex.get_distance()) {
            vertex.set_distance(best);
            vertex.set_updated(true);
            Medusa_Continue();
        } else {
            vertex.set_updated(false);
        }
    }
};

// an active source offers its distance plus the edge's weight
struct SendMsg {
    __device__ void operator()(D_Edge e, int super_step) {
        D_Vertex src(e.get_srcVertexID());
        if (src.get_updated()) e.sendMsg(src.get_distance() + e.get_weight());
    }
};
MEDUSA_BUILTIN_SSSP(SendMsg, distance, updated)

SendMsg sm;
UpdateVertex uv;
Message init_msg;

void Medusa_Exec() {
    init_msg.val = FLT_MAX;
    InitMessageBuffer(init_msg);
    FunctorHolder<EDGE>::Run(sm);
    MGLOBAL::com.combineAllDevice();
    FunctorHolder<VERTEX>::Run(uv);
}

int main(int argc, char **argv) {
    const dropin::Args a = dropin::parse(argc, argv);
    try {
        InitConfig("1", "0", EDGE_MESSAGE, false);
        MGLOBAL::rt.builtin_enabled = !a.generic;
        MGLOBAL::combiner_operator = CUDPP_MIN;
        MGLOBAL::combiner_datatype = CUDPP_FLOAT;
        InitHostDSFromGTGraph(a.graph);
        auto &va = MGLOBAL::gpu_def[0].vertexArray;
        for (int v = 0; v < va.size; v++) {
            va.distance[v] = MEDUSA_MAX;
            va.updated[v] = false;
        }
        va.distance[a.arg] = 0.0f;
        va.updated[a.arg] = true;
        InitDeviceDS();
        bool exe = true;
        while (exe) {
            ResetToExecute();
            Medusa_Exec();
            exe = RetriveToExecute();
            MGLOBAL::super_step++;
        }
        MGLOBAL::gpu_def[0].d_vertexArray.Dump(va);
        dropin::write_out(a.out, va.distance.data(), (size_t)va.size);
        dropin::report();
        MedusaShutdown();
    } catch (const std::exception &e) {
        std::fprintf(stderr, "dropin_sssp: %s\n", e.what());
        return 1;
    }
    return 0;
}
