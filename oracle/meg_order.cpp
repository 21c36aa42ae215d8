/*
 * meg_order.cpp -- the reference's MEG message order for the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY: linked into liboracle.so beside medusa_oracle.c;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
 *
 * The reference's PageRank app lays its edges out as MEG: GraphIR::sortByDegree
 * (MedusaRT/GraphConverter.cu:136-139) std::sorts the vertex records, in id
 * order, by descending out-degree (cmpVertexNode, :125-128), and
 * EdgeArray::buildMEG (MPG/EdgeDataType.cu:74-98) puts the k-th edge of the
 * vertex at sorted position i at position i + sum_{l<k} edgeOffset[l], where
 * edgeOffset[l] counts the vertices with more than l edges.  msgDstID then hands
 * out each destination's message slots in MEG position order (:121-123), so a
 * vertex's messages are summed in ascending MEG position of its in-edges.
 *
 * A vertex's k-th edge is its k-th edge in the AA order (the GraphIR edge list
 * is built by prepending, so both layouts walk it from the last edge added).
 * std::sort's permutation depends only on the outcomes of the comparisons, so
 * sorting (out-degree, id) records with the same comparison reproduces the
 * reference's order of equal-degree vertices.
 */
#include <stdint.h>

#include <algorithm>
#include <vector>

namespace {
struct Rec {
    int32_t deg, id;
};
}  // namespace

/* meg_slot[e], for AA edge e (edge_index / e_dst as orc_build_aa returns them):
 * the message slot of e in the reference's MEG order, with each destination's
 * slots at msg_index[v] .. msg_index[v+1]. */
extern "C" int orc_meg_slots(int32_t V, int64_t E, const int32_t *edge_index, const int32_t *e_dst,
                             const int32_t *msg_index, int32_t *meg_slot)
{
    try {
        std::vector<Rec> r((size_t)V);
        for (int32_t v = 0; v < V; v++) r[v] = Rec{edge_index[v + 1] - edge_index[v], v};
        std::sort(r.begin(), r.end(), [](const Rec &a, const Rec &b) { return a.deg > b.deg; });
        std::vector<int32_t> pos((size_t)V);
        for (int32_t i = 0; i < V; i++) pos[r[i].id] = i;
        const int32_t maxdeg = V ? r[0].deg : 0;
        // colstart[k] = sum_{l<k} edgeOffset[l]
        std::vector<int64_t> more((size_t)maxdeg + 1, 0), colstart((size_t)maxdeg + 1, 0);
        for (int32_t v = 0; v < V; v++)
            for (int32_t k = 0; k < edge_index[v + 1] - edge_index[v]; k++) more[k]++;
        for (int32_t k = 1; k <= maxdeg; k++) colstart[k] = colstart[k - 1] + more[k - 1];
        std::vector<int64_t> at_pos((size_t)(E > 0 ? E : 1));
        for (int32_t u = 0; u < V; u++)
            for (int32_t k = 0; k < edge_index[u + 1] - edge_index[u]; k++)
                at_pos[(size_t)(colstart[k] + pos[u])] = (int64_t)edge_index[u] + k;
        std::vector<int32_t> next(msg_index, msg_index + V);
        for (int64_t p = 0; p < E; p++) {
            const int64_t e = at_pos[(size_t)p];
            meg_slot[e] = next[e_dst[e]]++;
        }
    } catch (...) {
        return -1;
    }
    return 0;
}
