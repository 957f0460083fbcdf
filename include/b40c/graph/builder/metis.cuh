/*
 * METIS reader (drop-in for b40c/graph/builder/metis.cuh:193-230,
 * BuildMetisGraph / ReadMetisStream :51-187) over b40c_read_metis: "n m",
 * then one adjacency line per vertex (1-based ids); 2m ids expected (or m,
 * when the header counted every listed id).  Returns 0, or -1 after printing
 * the parse error.  With LOAD_VALUES every value is 1 (BFS reads none).
 */
#pragma once
#include "utils.cuh"
#include "file_utils.cuh"

namespace b40c {
namespace graph {
namespace builder {

template <bool LOAD_VALUES, typename VertexId, typename Value, typename SizeT>
int BuildMetisGraph(char *metis_filename, CsrGraph<VertexId, Value, SizeT> &csr_graph)
{
    b40c_csr g = {};
    if (b40c_read_metis(metis_filename, 0, &g) != 0) {
        fprintf(stderr, "%s\n", b40c_last_error_string());
        return -1;
    }
    return detail::AdoptFile<LOAD_VALUES>(g, csr_graph);
}

}  // namespace builder
}  // namespace graph
}  // namespace b40c
