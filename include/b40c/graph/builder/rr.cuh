/*
 * "Random-regular-ish" builder (drop-in for b40c/graph/builder/rr.cuh:53-91):
 * every vertex gets `degree` out-neighbours drawn with RandomNode (loops and
 * multi-edges possible, in-degrees not balanced), rows in vertex order.
 */
#pragma once
#include "utils.cuh"

namespace b40c {
namespace graph {
namespace builder {

template <bool LOAD_VALUES, typename VertexId, typename Value, typename SizeT>
int BuildRandomRegularishGraph(SizeT nodes, int degree, CsrGraph<VertexId, Value, SizeT> &csr_graph)
{
    const SizeT edges = nodes * degree;
    csr_graph.template FromScratch<LOAD_VALUES>(nodes, edges);
    printf("  Selecting %llu random edges in COO format... ", (unsigned long long)edges);
    fflush(stdout);
    time_t t0 = time(NULL);
    SizeT total = 0;
    for (SizeT node = 0; node < nodes; node++) {
        csr_graph.row_offsets[node] = total;
        for (int k = 0; k < degree; k++) {
            csr_graph.column_indices[total] = RandomNode(csr_graph.nodes);
            if (LOAD_VALUES) csr_graph.values[node] = 1;
            total++;
        }
    }
    csr_graph.row_offsets[nodes] = total;
    printf("Done selecting (%ds).\n", (int)(time(NULL) - t0));
    fflush(stdout);
    return 0;
}

}  // namespace builder
}  // namespace graph
}  // namespace b40c
