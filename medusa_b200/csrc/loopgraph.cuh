// loopgraph.cuh -- a whole BSP iteration loop as ONE CUDA graph launch.
//
// The reference runs its loop on the host: reset the device flag, launch the
// superstep's kernels, copy the flag back, repeat
// (MultipleGPU/MultiUtilities.h:48-69, SSSP/main.cu:369-382).  Here the loop
// lives on the device:
//
//   top graph:  prologue kernels  ->  WHILE(h_cont) {
//                                        select kernel (sets h_branch)
//                                        SWITCH(h_branch) { branch 0 .. n-1 }
//                                     }  ->  epilogue kernels
//
// The last CTA of every superstep kernel decides, on the device, whether to
// run another superstep and which branch it takes, and writes that to the
// control block.  The select kernel at the top of each iteration turns the
// control block into the two condition values: h_branch, and h_cont = 0 once
// the loop is done.  It also counts iterations and stops the loop past a
// hard cap, so the loop always ends.
#pragma once
#include <functional>
#include "mb_internal.cuh"

namespace mb {

struct LoopGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~LoopGraph() { reset(); }
};

using EmitFn = std::function<void(cudaStream_t)>;
using EmitSelect = std::function<void(cudaStream_t, cudaGraphConditionalHandle /*h_cont*/,
                                      cudaGraphConditionalHandle /*h_branch*/)>;
using EmitBranch = std::function<void(int, cudaStream_t)>;

inline void capture_into(cudaGraph_t g, const cudaGraphNode_t *deps, size_t ndeps,
                         cudaStream_t s, const EmitFn &emit) {
    MB_CUDA(cudaStreamBeginCaptureToGraph(s, g, deps, nullptr, ndeps,
                                          cudaStreamCaptureModeThreadLocal));
    try {
        emit(s);
    } catch (...) {
        cudaGraph_t tmp;
        cudaStreamEndCapture(s, &tmp);
        throw;
    }
    cudaGraph_t out = g;
    MB_CUDA(cudaStreamEndCapture(s, &out));
}

// Leaf nodes of g (nodes nothing depends on).
inline std::vector<cudaGraphNode_t> leaf_nodes(cudaGraph_t g) {
    size_t n = 0;
    MB_CUDA(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n), leaves;
    if (n) MB_CUDA(cudaGraphGetNodes(g, nodes.data(), &n));
    for (auto nd : nodes) {
        size_t nout = 0;
        MB_CUDA(cudaGraphNodeGetDependentNodes(nd, nullptr, &nout));
        if (nout == 0) leaves.push_back(nd);
    }
    return leaves;
}

inline void build_loop_graph(LoopGraph &lg, cudaStream_t s, int nbranch,
                             const EmitFn &prologue, const EmitSelect &select,
                             const EmitBranch &branch, const EmitFn &epilogue) {
    lg.reset();
    MB_CUDA(cudaGraphCreate(&lg.graph, 0));
    capture_into(lg.graph, nullptr, 0, s, prologue);
    std::vector<cudaGraphNode_t> deps = leaf_nodes(lg.graph);

    cudaGraphConditionalHandle h_cont;
    MB_CUDA(cudaGraphConditionalHandleCreate(&h_cont, lg.graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = h_cont;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    MB_CUDA(cudaGraphAddNode(&wnode, lg.graph, deps.data(), deps.size(), &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];

    cudaGraphConditionalHandle h_branch;
    MB_CUDA(cudaGraphConditionalHandleCreate(&h_branch, body, 0, 0));
    capture_into(body, nullptr, 0, s, [&](cudaStream_t st) { select(st, h_cont, h_branch); });
    std::vector<cudaGraphNode_t> bdeps = leaf_nodes(body);
    cudaGraphNodeParams sp = {};
    sp.type = cudaGraphNodeTypeConditional;
    sp.conditional.handle = h_branch;
    sp.conditional.type = cudaGraphCondTypeSwitch;
    sp.conditional.size = (unsigned)nbranch;
    cudaGraphNode_t snode;
    MB_CUDA(cudaGraphAddNode(&snode, body, bdeps.data(), bdeps.size(), &sp));
    for (int i = 0; i < nbranch; i++) {
        cudaGraph_t bg = sp.conditional.phGraph_out[i];
        capture_into(bg, nullptr, 0, s, [&](cudaStream_t st) { branch(i, st); });
    }
    if (epilogue) capture_into(lg.graph, &wnode, 1, s, epilogue);
    MB_CUDA(cudaGraphInstantiate(&lg.exec, lg.graph, 0));
}

}  // namespace mb
