/*
 * Shared tail of the file readers (market.cuh, dimacs.cuh, metis.cuh): moves a
 * graph parsed by the library (b40c_csr) into the caller's CsrGraph.
 */
#pragma once
#include <stdio.h>
#include <string.h>

#include "../csr_graph.cuh"
#include "b40c_bfs.h"

namespace b40c {
namespace graph {
namespace builder {
namespace detail {

template <bool LOAD_VALUES, typename VertexId, typename Value, typename SizeT>
int AdoptFile(b40c_csr &g, CsrGraph<VertexId, Value, SizeT> &csr_graph)
{
    csr_graph.template FromScratch<LOAD_VALUES>((SizeT)g.nodes, (SizeT)g.edges);
    memcpy(csr_graph.row_offsets, g.row_offsets, sizeof(SizeT) * (size_t)(g.nodes + 1));
    if (g.edges) memcpy(csr_graph.column_indices, g.column_indices, sizeof(VertexId) * (size_t)g.edges);
    if (LOAD_VALUES)
        for (long long e = 0; e < g.edges; e++) csr_graph.values[e] = 1;
    b40c_graph_free(&g);
    return 0;
}

}  // namespace detail
}  // namespace builder
}  // namespace graph
}  // namespace b40c
