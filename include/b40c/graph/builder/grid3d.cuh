/*
 * 3D lattice builder (drop-in for b40c/graph/builder/grid3d.cuh:54-129):
 * width^3 vertices, id = (z * width + y) * width + x, neighbours in the order
 * -x, +x, -y, +y, -z, +z, then a self-loop.  Returns 0, or -1 on a negative width.
 */
#pragma once
#include "utils.cuh"

namespace b40c {
namespace graph {
namespace builder {

template <bool LOAD_VALUES, typename VertexId, typename Value, typename SizeT>
int BuildGrid3dGraph(VertexId width, CsrGraph<VertexId, Value, SizeT> &csr_graph)
{
    if (width < 0) {
        fprintf(stderr, "Invalid width: %lld", (long long)width);
        return -1;
    }
    const SizeT w = width, nodes = w * w * w;
    const SizeT edges = nodes + (w > 1 ? 6 * w * w * (w - 1) : 0);
    csr_graph.template FromScratch<LOAD_VALUES>(nodes, edges);
    const VertexId plane = width * width;
    SizeT total = 0;
    for (VertexId z = 0; z < width; z++)
        for (VertexId y = 0; y < width; y++)
            for (VertexId x = 0; x < width; x++) {
                const VertexId me = z * plane + y * width + x;
                csr_graph.row_offsets[me] = total;
                const VertexId nbr[6] = {me - 1, me + 1, me - width, me + width, me - plane, me + plane};
                const bool ok[6] = {x > 0, x + 1 < width, y > 0, y + 1 < width, z > 0, z + 1 < width};
                for (int k = 0; k < 6; k++)
                    if (ok[k]) csr_graph.column_indices[total++] = nbr[k];
                csr_graph.column_indices[total++] = me;
                if (LOAD_VALUES) csr_graph.values[me] = 1;
            }
    csr_graph.row_offsets[nodes] = total;
    return 0;
}

}  // namespace builder
}  // namespace graph
}  // namespace b40c
