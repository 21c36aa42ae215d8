// multigraph.cuh -- many independent graphs in one persistent launch (internal).
#pragma once
#include <vector>
#include "mb_internal.cuh"

namespace mb {

// Per-graph descriptor read by the persistent kernel.
struct GDesc {
    int32_t V;
    int32_t E;
    const int32_t *row, *col, *rrow, *rcol;  // the graph's own arrays (local ids)
    int64_t vbase;                           // offset in the batch-wide vertex arrays
    int32_t team;                            // CTAs that run this graph together
    int32_t source;                          // BFS source (set per run)
};

// Shared state of one graph's team (zeroed before each run).
struct TeamState {
    unsigned bar_count, bar_gen;     // team barrier
    unsigned qn[3];                  // BFS queue counters, rotating by level
    int32_t pad;
    unsigned long long reached_edges;  // BFS: out-edges of reached vertices
    unsigned long long reached;        // BFS: reached vertices
};

struct Batch {
    std::vector<Graph> graphs;        // built with the single-graph builder
    std::vector<int64_t> vbase;       // n+1 prefix of vertex counts
    int64_t total_V = 0, total_E = 0;
    DevBuf desc, team, entries, contrib[2], queue[2], rank, level, work;
    int32_t nentries = 0;
    int64_t desc_gen = -1;            // tunables generation the entries were built for
    ~Batch() { release(); }
    void release() {
        for (auto &g : graphs) g.release();
        graphs.clear();
        desc.release(); team.release(); entries.release();
        contrib[0].release(); contrib[1].release(); queue[0].release(); queue[1].release();
        rank.release(); level.release(); work.release();
    }
};

// Build the batch's graphs (reference order) from generator parameters.
void batch_generate(Context &ctx, Batch &b, const mb_gen_params *params, int32_t n);
// Build the batch's graphs (reference order) from the caller's edge lists:
// graph i has nv[i] vertices and the ne[i] edges that follow graph i-1's in
// src / dst (host or device memory), with ids local to the graph.
void batch_from_edges(Context &ctx, Batch &b, int32_t n, const int32_t *nv, const int64_t *ne,
                      const int32_t *src, const int32_t *dst);
// The batch's work buffers, after its graphs are built.
void batch_finish(Batch &b);

// One persistent cooperative launch: for every graph, `pr_iters` PageRank
// supersteps from 1/V_g, then one BFS from sources[g] (nullptr: vertex 0).
// Ranks and levels of graph g land at [vbase[g], vbase[g+1]) of the outputs
// (device pointers).
void batch_run(Context &ctx, Batch &b, int32_t pr_iters, const int32_t *sources, float *ranks_dev,
               int32_t *levels_dev, mb_stats *stats);

}  // namespace mb
