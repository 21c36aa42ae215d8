// dropin_bfs.cu -- the reference's BFS app (Algorithm/Vertex.h,
// Algorithm/UserOperators.h:17-52, Algorithm/main.cu:224-300) as it compiles
// against include/medusa/medusa.h: the level attribute becomes a field list
// entry, the edge functor and the BSP loop keep their shape, and one line
// routes the functor to the library's BFS (mb_bfs).
#define MEDUSA_VERTEX_FIELDS(F) F(int, level)
#include <medusa/medusa.h>

#include "dropin_common.h"

#define MVT_Init_Value -1

// a frontier vertex (level == super_step) reaches its unvisited neighbours
struct UpdateLevel {
    __device__ void operator()(D_Edge e, int super_step) {
        D_Vertex src(e.get_srcVertexID());
        if (src.get_level() == super_step) {
            D_Vertex dst(e.get_dstVertexID());
            if (dst.get_level() == MVT_Init_Value) {
                dst.set_level(super_step + 1);
                Medusa_Continue();
            }
        }
    }
};
MEDUSA_BUILTIN_BFS(UpdateLevel, level)

UpdateLevel ul;

void Medusa_Exec() { FunctorHolder<EDGE>::Run(ul); }

int main(int argc, char **argv) {
    const dropin::Args a = dropin::parse(argc, argv);
    try {
        InitConfig("1", "0", NO_MESSAGE, false);
        MGLOBAL::rt.builtin_enabled = !a.generic;
        InitHostDSFromGTGraph(a.graph);
        auto &va = MGLOBAL::gpu_def[0].vertexArray;
        for (int v = 0; v < va.size; v++) va.level[v] = MVT_Init_Value;
        va.level[a.arg] = 0;
        InitDeviceDS();
        bool exe = true;
        while (exe) {
            ResetToExecute();
            Medusa_Exec();
            exe = RetriveToExecute();
            MGLOBAL::super_step++;
        }
        MGLOBAL::gpu_def[0].d_vertexArray.Dump(va);
        dropin::write_out(a.out, va.level.data(), (size_t)va.size);
        dropin::report();
        MedusaShutdown();
    } catch (const std::exception &e) {
        std::fprintf(stderr, "dropin_bfs: %s\n", e.what());
        return 1;
    }
    return 0;
}
