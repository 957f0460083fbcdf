/*
 * DIMACS reader (drop-in for b40c/graph/builder/dimacs.cuh:235-283,
 * BuildDimacsGraph / ReadDimacsStream :52-228) over b40c_read_dimacs:
 * "p <type> n m" then "a u v [w]" arcs, 1-based; splice > 0 merges the files
 * <name>.0, <name>.1, ... by smallest row; reverse edges when undirected.
 * Returns 0, or -1 after printing the parse error.  With LOAD_VALUES every
 * value is 1 (BFS reads none).
 */
#pragma once
#include "utils.cuh"
#include "file_utils.cuh"

namespace b40c {
namespace graph {
namespace builder {

template <bool LOAD_VALUES, typename VertexId, typename Value, typename SizeT>
int BuildDimacsGraph(char *dimacs_filename, CsrGraph<VertexId, Value, SizeT> &csr_graph, bool undirected, int splice)
{
    b40c_csr g = {};
    if (b40c_read_dimacs(dimacs_filename, undirected ? 1 : 0, splice, 0, &g) != 0) {
        fprintf(stderr, "%s\n", b40c_last_error_string());
        return -1;
    }
    return detail::AdoptFile<LOAD_VALUES>(g, csr_graph);
}

}  // namespace builder
}  // namespace graph
}  // namespace b40c
