// vis.cu -- the reference's visualisation coordinates, into a headless
// device buffer instead of OpenGL vertex buffers (no graphics stack here).
//
// DrawNodes (MedusaRT/GraphRenderingAPI.cu:33-44): vertex v with centre
// (x, y) and integer radius r gets the quad
//   (x - r, y + r - 1), (x + r - 1, y + r - 1), (x + r - 1, y - r), (x - r, y - r)
// DrawEdges (:69-78): edge e gets the endpoints pos[src(e)], pos[dst(e)], in
// the reference's edge-array order (the CSR's AA order).
// Each vertex's quad is two 16-byte stores and each edge's line one, so the
// output streams at full width; the edge kernel's position reads are
// gathers (8 bytes per endpoint).
#include "mb_internal.cuh"

namespace mb {
namespace {

__global__ void k_node_quads(int32_t V, const float2 *__restrict__ pos, const int32_t *__restrict__ radius,
                             float4 *__restrict__ quads) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V;
         v += (int64_t)gridDim.x * blockDim.x) {
        const float2 c = pos[v];
        const int r = radius[v];
        // the reference's float2 arithmetic: int radius converted per term
        quads[2 * v] = make_float4(c.x - r, c.y + r - 1, c.x + r - 1, c.y + r - 1);
        quads[2 * v + 1] = make_float4(c.x + r - 1, c.y - r, c.x - r, c.y - r);
    }
}

__global__ void k_edge_lines(int64_t E, const int32_t *__restrict__ esrc, const int32_t *__restrict__ col,
                             const float2 *__restrict__ pos, float4 *__restrict__ lines) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E;
         e += (int64_t)gridDim.x * blockDim.x) {
        const float2 a = pos[esrc[e]], b = pos[col[e]];
        lines[e] = make_float4(a.x, a.y, b.x, b.y);
    }
}

}  // namespace

void vis_node_quads(Context &ctx, int32_t V, const float *pos, const int32_t *radius, float *quads) {
    if (V <= 0) return;
    k_node_quads<<<grid_for(V, 256, ctx.num_sms * 16), 256, 0, ctx.stream>>>(
        V, (const float2 *)pos, radius, (float4 *)quads);
    MB_CHECK_LAUNCH();
}

void vis_edge_lines(Context &ctx, const Graph &g, const float *pos, float *lines) {
    if (g.E <= 0) return;
    k_edge_lines<<<grid_for(g.E, 256, ctx.num_sms * 16), 256, 0, ctx.stream>>>(
        g.E, g.esrc.as<int32_t>(), g.col.as<int32_t>(), (const float2 *)pos, (float4 *)lines);
    MB_CHECK_LAUNCH();
}

}  // namespace mb
