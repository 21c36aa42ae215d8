// apps_main.cu -- command-line driver of the operator-API apps:
//
//   medusa_apps bfs|sssp|pr|prmsg <gtgraph file> <source | supersteps> <output file>
//
// Reads the graph with InitHostDSFromGTGraph (GPU GTgraph parser), runs the
// app through the generic functor kernels of include/medusa/medusa.h and
// writes the raw int32 levels / float32 distances / float32 ranks.
#include <cstdio>
#include <cstdlib>
#include "bfs_ops.cuh"
#include "msg_ops.cuh"
#include "pagerank_ops.cuh"
#include "sssp_ops.cuh"

template <class T>
static void write_out(const char *path, const std::vector<T> &v) {
    FILE *f = std::fopen(path, "wb");
    if (!f) throw std::runtime_error(std::string("cannot write ") + path);
    std::fwrite(v.data(), sizeof(T), v.size(), f);
    std::fclose(f);
}

int main(int argc, char **argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: medusa_apps bfs|sssp|pr|prmsg <gtgraph file> <source|supersteps> <out>\n");
        return 2;
    }
    try {
        const std::string app = argv[1];
        const int arg = std::atoi(argv[3]);
        InitConfig("1", "0", EDGE_MESSAGE, false);
        InitHostDSFromGTGraph(argv[2]);
        if (app == "bfs") write_out(argv[4], bfs_app::run(arg));
        else if (app == "sssp") write_out(argv[4], sssp_app::run(arg));
        else if (app == "pr") write_out(argv[4], pagerank_app::run(arg));
        else if (app == "prmsg") write_out(argv[4], msg_app::run(arg));
        else throw std::runtime_error("unknown app " + app);
        std::printf("%s done: %d supersteps\n", app.c_str(), MGLOBAL::super_step);
        MedusaShutdown();
    } catch (const std::exception &e) {
        std::fprintf(stderr, "medusa_apps: %s\n", e.what());
        return 1;
    }
    return 0;
}
