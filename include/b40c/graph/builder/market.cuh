/*
 * MARKET reader (drop-in for b40c/graph/builder/market.cuh:180-208,
 * BuildMarketGraph / ReadMarketStream :49-160) over the library's native
 * parser b40c_read_market: "rows cols nnz" then "col row [value]" lines,
 * 1-based, reverse edges when undirected, rows in file order.  Returns 0, or
 * -1 after printing the parse error.  With LOAD_VALUES every value is 1
 * (BFS reads none).
 */
#pragma once
#include "utils.cuh"
#include "file_utils.cuh"

namespace b40c {
namespace graph {
namespace builder {

template <bool LOAD_VALUES, typename VertexId, typename Value, typename SizeT>
int BuildMarketGraph(char *market_filename, CsrGraph<VertexId, Value, SizeT> &csr_graph, bool undirected)
{
    b40c_csr g = {};
    if (b40c_read_market(market_filename, undirected ? 1 : 0, 0, &g) != 0) {
        fprintf(stderr, "%s\n", b40c_last_error_string());
        return -1;
    }
    return detail::AdoptFile<LOAD_VALUES>(g, csr_graph);
}

}  // namespace builder
}  // namespace graph
}  // namespace b40c
