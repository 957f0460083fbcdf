/*
 * COO edge tuple (drop-in for b40c/graph/coo_edge_tuple.cuh:52-100): fields
 * row, col (and val unless Value is util::NullType), and the by-row
 * comparator CsrGraph::FromCoo sorts with.
 */
#pragma once
#include "../util/basic_utils.cuh"

namespace b40c {
namespace graph {

template <typename VertexId, typename Value>
struct CooEdgeTuple {
    VertexId row;
    VertexId col;
    Value val;

    CooEdgeTuple() {}
    CooEdgeTuple(VertexId row, VertexId col, Value val) : row(row), col(col), val(val) {}
    void Val(Value &value) { value = val; }
};

template <typename VertexId>
struct CooEdgeTuple<VertexId, util::NullType> {
    VertexId row;
    VertexId col;

    CooEdgeTuple() {}
    template <typename Value>
    CooEdgeTuple(VertexId row, VertexId col, Value) : row(row), col(col) {}
    template <typename Value>
    void Val(Value &) {}
};

/* Orders edges by source row only, so a stable sort keeps each row's edges in
 * their original order. */
template <typename Tuple>
bool DimacsTupleCompare(Tuple a, Tuple b)
{
    return a.row < b.row;
}

}  // namespace graph
}  // namespace b40c
