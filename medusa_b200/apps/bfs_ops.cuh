// bfs_ops.cuh -- BFS written against the operator API (include/medusa/medusa.h),
// in the shape of the reference's Algorithm/UserOperators.h:17-35 and
// Algorithm/main.cu:225-300: one EDGE functor per superstep, no messages.
#pragma once
#include <medusa/medusa.h>

namespace bfs_app {

// UpdateLevel: an edge whose source was reached at this superstep reaches its
// destination at the next one (level -1: not reached).
struct UpdateLevel {
    int *level;
    __device__ void operator()(D_Edge e, int super_step) {
        if (level[e.get_srcVertexID()] == super_step) {
            const int dst = e.get_dstVertexID();
            if (level[dst] == -1) {
                level[dst] = super_step + 1;
                Medusa_Continue();
            }
        }
    }
};

inline void Medusa_Exec(UpdateLevel &ul) { FunctorHolder<EDGE>::Run(ul); }

// Levels from `source` on the graph InitHostDS built.
inline std::vector<int> run(int source) {
    InitConfig("1", "0", NO_MESSAGE, false);
    InitDeviceDS();
    const int V = MGLOBAL::rt.view.num_vertices;
    medusa::DeviceArray<int> level(V);
    std::vector<int> h(V, -1);
    h[source] = 0;
    level.upload(h.data());
    UpdateLevel ul{level.data()};
    bool exe = true;
    while (exe) {
        ResetToExecute();
        Medusa_Exec(ul);
        exe = RetriveToExecute();
        MGLOBAL::super_step++;
    }
    return level.to_host();
}

}  // namespace bfs_app
