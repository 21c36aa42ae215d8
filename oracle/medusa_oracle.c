/*
 * medusa_oracle.c -- CPU restatement of Medusa's single-GPU BSP superstep.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * medusa_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  Nothing in the product links or calls it.
 *
 * It restates, in plain C, what the reference computes for the three apps on
 * its hot path, in the reference's own (synchronous, edge-centric) form:
 *
 *   layout   GraphIR::AddEdge          MedusaRT/GraphConverter.cu:180-196
 *            VertexArray::build        SSSP/VertexDataType.cu:64-85
 *            EdgeArray::buildAA        SSSP/EdgeDataType.cu:138-186
 *   BFS      BFS_Edge_Processor        Algorithm/CPUFunctorHoster.cpp:16-30
 *            Medusa_Exec_CPU           Algorithm/CPUFunctorHoster.cpp:35-65
 *   SSSP     SSSP_Edge_Processor_SendMsg     SSSP/CPUFunctorHoster.cpp:40-49
 *            SSSP_Vertex_Processor_UpdateVertex SSSP/CPUFunctorHoster.cpp:15-33
 *            Medusa_Exec_CPU           SSSP/CPUFunctorHoster.cpp:58-99
 *   PageRank PG_Vertex_Processor_SendMsg     MPG/CPUFunctorHoster.cpp:60-93 (AA branch)
 *            PG_Vertex_Processor_UpdateVertex MPG/CPUFunctorHoster.cpp:17-31
 *            Medusa_Exec_CPU loop      MPG/CPUFunctorHoster.cpp:143-163
 *
 * Parity is pinned: tests/golden/ holds outputs of the reference's own CPU
 * code (compiled from its sources by oracle/ref/build_ref.py) on seeded
 * graphs, and tests/test_oracle.py checks this file against them.
 *
 * Sentinels follow the reference: BFS unreached level = -1
 * (Algorithm/Message.h:10), SSSP unreached distance = MEDUSA_MAX = 1e9
 * (SSSP/Configuration.h:6, SSSP/main.cu:324), SSSP message identity FLT_MAX
 * (SSSP/CPUFunctorHoster.cpp:68), PageRank message identity 0
 * (MPG/CPUFunctorHoster.cpp:152).
 */
#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MEDUSA_MAX 1000000000.0f

/*
 * AA layout of an edge list given in insertion order.
 *
 * GraphIR::AddEdge prepends each edge to its source's list
 * (GraphConverter.cu:191-192), and buildAA walks every list from its head
 * (SSSP/EdgeDataType.cu:148-157), so within one source the AA order is the
 * REVERSE of insertion order.  A counting sort by source that visits the
 * edges from last to first produces exactly that order.
 *
 * Outputs (caller-allocated):
 *   edge_index[V+1]  prefix of out-degrees      (SSSP/VertexDataType.cu:79-83)
 *   msg_index[V+1]   prefix of in-degrees       (SSSP/VertexDataType.cu:75-77)
 *   e_src/e_dst/e_w[E] edges in AA order
 *   msg_dst[E]       slot of the edge's message in the dst-grouped message
 *                    array: a per-destination cursor advanced in AA order
 *                    (SSSP/EdgeDataType.cu:181-182)
 *   perm[E]          input index of each AA edge (nullable)
 * Returns 0, or -1 on a bad id / allocation failure.
 */
int orc_build_aa(int32_t V, int64_t E, const int32_t *src, const int32_t *dst,
                 const float *w, int32_t *edge_index, int32_t *msg_index,
                 int32_t *e_src, int32_t *e_dst, float *e_w, int32_t *msg_dst,
                 int64_t *perm)
{
    int64_t *cur = (int64_t *)calloc((size_t)V + 1, sizeof(int64_t));
    int64_t *mcur = (int64_t *)calloc((size_t)V + 1, sizeof(int64_t));
    if (!cur || !mcur) { free(cur); free(mcur); return -1; }
    for (int64_t e = 0; e < E; e++) {
        if (src[e] < 0 || src[e] >= V || dst[e] < 0 || dst[e] >= V) {
            free(cur); free(mcur); return -1;
        }
        cur[src[e] + 1]++;
        mcur[dst[e] + 1]++;
    }
    for (int32_t v = 0; v < V; v++) { cur[v + 1] += cur[v]; mcur[v + 1] += mcur[v]; }
    for (int32_t v = 0; v <= V; v++) { edge_index[v] = (int32_t)cur[v]; msg_index[v] = (int32_t)mcur[v]; }
    /* place: last inserted edge of a source first */
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * ((size_t)V + 1));
    if (!fill) { free(cur); free(mcur); return -1; }
    memcpy(fill, cur, sizeof(int64_t) * ((size_t)V + 1));
    for (int64_t e = E - 1; e >= 0; e--) {
        int64_t p = fill[src[e]]++;
        e_src[p] = src[e];
        e_dst[p] = dst[e];
        e_w[p] = w ? w[e] : 0.0f;
        if (perm) perm[p] = e;
    }
    for (int64_t p = 0; p < E; p++) msg_dst[p] = (int32_t)(mcur[e_dst[p]]++);
    free(fill); free(cur); free(mcur);
    return 0;
}

/*
 * BFS, edge-centric over all edges every superstep
 * (Algorithm/CPUFunctorHoster.cpp:16-30, loop :35-65).  level[] must hold -1
 * everywhere and 0 at the sources on entry (Algorithm/main.cu:225-254).
 * Returns the number of supersteps run, the last one being the step that
 * changed nothing, as the reference counts them (:53-62).
 */
int orc_bfs(int32_t V, int64_t E, const int32_t *e_src, const int32_t *e_dst,
            int32_t *level)
{
    (void)V;
    int step = 0;
    for (;;) {
        int cont = 0;
        for (int64_t e = 0; e < E; e++) {
            if (level[e_src[e]] == step) {
                int32_t d = e_dst[e];
                if (level[d] == -1) { level[d] = step + 1; cont = 1; }
            }
        }
        step++;
        if (!cont) break;
    }
    return step;
}

/*
 * SSSP as the reference's CPU path runs it: synchronous Bellman-Ford.  Every
 * superstep resets the E-slot message array to FLT_MAX, every edge writes
 * dist[src]+w into its slot (the "updated" filter is commented out at
 * SSSP/CPUFunctorHoster.cpp:44-48), then each vertex takes the minimum of its
 * slots and lowers its distance (:15-33).  dist[] must hold 1e9 everywhere and
 * 0 at the source on entry (SSSP/main.cu:322-352).  Returns supersteps run.
 */
int orc_sssp(int32_t V, int64_t E, const int32_t *e_src, const float *e_w,
             const int32_t *msg_dst, const int32_t *msg_index, float *dist)
{
    float *msg = (float *)malloc(sizeof(float) * (size_t)(E > 0 ? E : 1));
    if (!msg) return -1;
    int step = 0;
    for (;;) {
        int cont = 0;
        for (int64_t e = 0; e < E; e++) msg[e] = FLT_MAX;
        for (int64_t e = 0; e < E; e++) msg[msg_dst[e]] = dist[e_src[e]] + e_w[e];
        for (int32_t v = 0; v < V; v++) {
            float m = FLT_MAX;
            for (int32_t i = msg_index[v]; i < msg_index[v + 1]; i++)
                if (msg[i] < m) m = msg[i];
            if (m < dist[v]) { dist[v] = m; cont = 1; }
        }
        step++;
        if (!cont) break;
    }
    free(msg);
    return step;
}

/*
 * The GPU's fixed summation order for a vertex's n messages m[0..n) (slot
 * order): n <= 64, a sequential fold; else blocks of 4096 messages, each the
 * 32-lane strided fold (lane l: m[l], m[l+32], ... in order) reduced by an
 * xor butterfly (each step t[l] = s[l] + s[l ^ off], off = 16, 8, 4, 2, 1),
 * the block results folded sequentially.  Not the reference's order: the
 * reference folds sequentially (MPG/CPUFunctorHoster.cpp:21-26); this order
 * is what the CUDA kernels compute, so they can be checked bit for bit.
 */
#define ORC_PR_LIGHT 64
#define ORC_PR_BLOCK 4096
static float orc_fold_blocked(const float *m, int32_t n)
{
    float total = 0.0f;
    if (n <= ORC_PR_LIGHT) {
        for (int32_t i = 0; i < n; i++) total += m[i];
        return total;
    }
    for (int32_t b0 = 0; b0 < n; b0 += ORC_PR_BLOCK) {
        int32_t b1 = n < b0 + ORC_PR_BLOCK ? n : b0 + ORC_PR_BLOCK;
        float lane[32], t[32];
        for (int l = 0; l < 32; l++) {
            lane[l] = 0.0f;
            for (int32_t j = b0 + l; j < b1; j += 32) lane[l] += m[j];
        }
        for (int off = 16; off; off >>= 1) {
            for (int l = 0; l < 32; l++) t[l] = lane[l] + lane[l ^ off];
            for (int l = 0; l < 32; l++) lane[l] = t[l];
        }
        total += lane[0];
    }
    return total;
}

/*
 * PageRank in the reference's non-normalised form, FP32, with the reference's
 * mixed-precision update: sum is float, "sum *= 0.85" multiplies by a double
 * literal and rounds back to float, "0.15 + sum" adds in double and rounds to
 * float (MPG/CPUFunctorHoster.cpp:21-29).  msg = rank/out_degree in float
 * (:80-82).  order 0: each vertex sums its slots sequentially in msg_index
 * order (the reference's fold); order 1: the GPU's fixed order
 * (orc_fold_blocked).  iters supersteps, rank[] holds the initial ranks on
 * entry.
 */
int orc_pagerank_f32(int32_t V, int64_t E, const int32_t *e_src,
                     const int32_t *msg_dst, const int32_t *msg_index,
                     const int32_t *edge_index, int iters, float *rank, int order)
{
    float *msg = (float *)malloc(sizeof(float) * (size_t)(E > 0 ? E : 1));
    if (!msg) return -1;
    /* Every slot and every vertex is written by one OpenMP thread, and each
     * vertex's fold runs in one thread in its own order, so the bits do not
     * depend on the thread count. */
    for (int it = 0; it < iters; it++) {
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < E; e++) {
            int32_t s = e_src[e];
            int32_t cnt = edge_index[s + 1] - edge_index[s];
            msg[msg_dst[e]] = rank[s] / (float)cnt;
        }
#pragma omp parallel for schedule(dynamic, 4096)
        for (int32_t v = 0; v < V; v++) {
            float sum = 0.0f;
            if (order == 1) {
                sum = orc_fold_blocked(msg + msg_index[v], msg_index[v + 1] - msg_index[v]);
            } else {
                for (int32_t i = msg_index[v]; i < msg_index[v + 1]; i++) sum += msg[i];
            }
            sum = (float)((double)sum * 0.85);
            rank[v] = (float)(0.15 + (double)sum);
        }
    }
    free(msg);
    return iters;
}

/* The same PageRank in FP64 throughout: the accuracy yardstick for both the
 * reference FP32 result and the GPU FP32 result.  The scatter and the
 * per-vertex sums are split over OpenMP threads (each message slot and each
 * vertex is written by one thread, so the result does not depend on the
 * thread count). */
int orc_pagerank_f64(int32_t V, int64_t E, const int32_t *e_src,
                     const int32_t *msg_dst, const int32_t *msg_index,
                     const int32_t *edge_index, int iters, double *rank)
{
    double *msg = (double *)malloc(sizeof(double) * (size_t)(E > 0 ? E : 1));
    if (!msg) return -1;
    for (int it = 0; it < iters; it++) {
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < E; e++) {
            int32_t s = e_src[e];
            msg[msg_dst[e]] = rank[s] / (double)(edge_index[s + 1] - edge_index[s]);
        }
#pragma omp parallel for schedule(dynamic, 4096)
        for (int32_t v = 0; v < V; v++) {
            double sum = 0.0;
            for (int32_t i = msg_index[v]; i < msg_index[v + 1]; i++) sum += msg[i];
            rank[v] = 0.15 + 0.85 * sum;
        }
    }
    free(msg);
    return iters;
}
