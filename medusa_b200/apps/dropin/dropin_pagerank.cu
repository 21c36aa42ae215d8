// dropin_pagerank.cu -- the reference's PageRank app (MPG/Vertex.h,
// MPG/UserOperators.h:16-43,175-270, MPG/main.cu:120-169) as it compiles
// against include/medusa/medusa.h: the rank attribute (the reference calls
// it "level") becomes a field list entry, the functors and the loop keep
// their shape, and one line routes each superstep to the library's PageRank
// (mb_pagerank_from, one superstep per Medusa_Exec).
#define MEDUSA_VERTEX_FIELDS(F) F(MVT, level)
#include <medusa/medusa.h>

#include "dropin_common.h"

struct Message {
    MVT val;
};

// rank = 0.15 + 0.85 * (sum of the in-neighbours' rank / out-degree)
struct UpdateVertex {
    __device__ void operator()(D_Vertex vertex, int super_step) {
        MVT sum = vertex.get_combined_msg();
        sum *= 0.85;
        vertex.set_level(0.15 + sum);
    }
};

// every vertex sends its rank shared out over its out-edges
struct SendMsg {
    __device__ void operator()(D_Edge e, int super_step) {
        D_Vertex src(e.get_srcVertexID());
        e.sendMsg(src.get_level() / src.get_edge_count());
    }
};
MEDUSA_BUILTIN_PAGERANK(SendMsg, level)

SendMsg sm;
UpdateVertex uv;
Message init_msg;

void Medusa_Exec() {
    init_msg.val = 0;
    InitMessageBuffer(init_msg);
    FunctorHolder<EDGE>::Run(sm);
    MGLOBAL::com.combineAllDevice();
    FunctorHolder<VERTEX>::Run(uv);
}

int main(int argc, char **argv) {
    const dropin::Args a = dropin::parse(argc, argv);
    try {
        InitConfig("1", "0", EDGE_MESSAGE, true);
        MGLOBAL::rt.builtin_enabled = !a.generic;
        MGLOBAL::combiner_operator = CUDPP_ADD;
        MGLOBAL::combiner_datatype = CUDPP_FLOAT;
        InitHostDSFromGTGraph(a.graph);
        auto &va = MGLOBAL::gpu_def[0].vertexArray;
        for (int v = 0; v < va.size; v++) va.level[v] = 1.0f / (float)va.size;
        InitDeviceDS();
        bool exe = true;
        while (exe) {
            Medusa_Exec();
            exe = RetriveToExecute();
            MGLOBAL::super_step++;
            if (MGLOBAL::super_step >= a.arg) break;  // the app's fixed number of supersteps
        }
        MGLOBAL::gpu_def[0].d_vertexArray.Dump(va);
        dropin::write_out(a.out, va.level.data(), (size_t)va.size);
        dropin::report();
        MedusaShutdown();
    } catch (const std::exception &e) {
        std::fprintf(stderr, "dropin_pagerank: %s\n", e.what());
        return 1;
    }
    return 0;
}
