// dropin_common.h -- the driver shared by the drop-in apps: the command line,
// the output file and the report of which path ran.
//
//   medusa_dropin_<app> <gtgraph file> <source | supersteps> <output file> [generic]
//
// "generic" turns the built-in routing off, so the same functors run through
// the generic FunctorHolder kernels.  stdout ends with one line
//   path=<builtin app id> generic_launches=<n> kernel_launches=<n> supersteps=<n> schedules=<8 counts>
// (the library's statistics of the routed call).
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace dropin {

struct Args {
    std::string graph, out;
    int arg = 0;
    bool generic = false;
};

inline Args parse(int argc, char **argv) {
    if (argc < 4 || argc > 5 || (argc == 5 && std::strcmp(argv[4], "generic") != 0)) {
        std::fprintf(stderr, "usage: %s <gtgraph file> <source|supersteps> <out> [generic]\n", argv[0]);
        std::exit(2);
    }
    Args a;
    a.graph = argv[1];
    a.arg = std::atoi(argv[2]);
    a.out = argv[3];
    a.generic = argc == 5;
    return a;
}

template <class T>
inline void write_out(const std::string &path, const T *p, size_t n) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fwrite(p, sizeof(T), n, f);
    std::fclose(f);
}

inline void report() {
    const auto &rt = MGLOBAL::rt;
    std::printf("path=%d generic_launches=%lld kernel_launches=%lld supersteps=%d schedules=",
                (int)rt.last_builtin, (long long)rt.generic_launches,
                (long long)rt.builtin_stats.kernel_launches, rt.builtin_stats.supersteps);
    for (int i = 0; i < MB_NUM_SCHEDULES; i++)
        std::printf("%s%d", i ? "," : "", rt.builtin_stats.schedule_count[i]);
    std::printf("\n");
}

}  // namespace dropin
