/*
 * Uniform random graph builder (drop-in for b40c/graph/builder/random.cuh:54-98):
 * `edges` (RandomNode, RandomNode) pairs, each followed by its reverse when
 * `undirected`, loops and multi-edges kept; libc rand() in the reference's order.
 */
#pragma once
#include "utils.cuh"

namespace b40c {
namespace graph {
namespace builder {

template <bool LOAD_VALUES, typename VertexId, typename Value, typename SizeT>
int BuildRandomGraph(SizeT nodes, SizeT edges, CsrGraph<VertexId, Value, SizeT> &csr_graph, bool undirected)
{
    typedef CooEdgeTuple<VertexId, Value> EdgeTupleType;
    if (nodes < 0 || edges < 0) {
        fprintf(stderr, "Invalid graph size: nodes=%lld, edges=%lld", (long long)nodes, (long long)edges);
        return -1;
    }
    printf("  Selecting %llu %s random edges in COO format... ", (unsigned long long)edges,
           undirected ? "undirected" : "directed");
    fflush(stdout);
    time_t t0 = time(NULL);
    const SizeT directed_edges = undirected ? edges * 2 : edges;
    EdgeTupleType *coo = (EdgeTupleType *)malloc(sizeof(EdgeTupleType) * (size_t)(directed_edges > 0 ? directed_edges : 1));
    if (!coo) {
        fprintf(stderr, "BuildRandomGraph: out of memory\n");
        return -1;
    }
    for (SizeT i = 0; i < edges; i++) {
        const VertexId u = RandomNode(nodes);
        const VertexId v = RandomNode(nodes);
        coo[i] = EdgeTupleType(u, v, 1);
        if (undirected) coo[edges + i] = EdgeTupleType(v, u, 1);
    }
    printf("Done selecting (%ds).\n", (int)(time(NULL) - t0));
    fflush(stdout);
    csr_graph.template FromCoo<LOAD_VALUES>(coo, nodes, directed_edges);
    free(coo);
    return 0;
}

}  // namespace builder
}  // namespace graph
}  // namespace b40c
