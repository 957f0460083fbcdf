/*
 * R-MAT builder (drop-in for b40c/graph/builder/rmat.cuh:45-206).
 *
 * Each of `edges` edges walks the adjacency matrix from (1, 1) down log2(nodes)
 * levels, picking a quadrant with probabilities a, b, c, d = 1 - a - b - c,
 * which are perturbed by up to 5% and renormalised after every level; with
 * `undirected` each edge also gets its reverse.  Self-loops and duplicates
 * are kept.  Random numbers come from libc rand() in the reference's order
 * (one draw per quadrant choice, then per parameter a sign draw and a
 * magnitude draw), so the same srand() seed gives the same graph.
 *
 * One difference: the walk starts at id 1, so a walk that takes the last
 * quadrant's half at every level ends at id `nodes`, one past the last vertex
 * (the reference keeps it: its CSR then ends short of `edges` and indexes past
 * its arrays).  Such an id wraps to 0 here, as in the library's native
 * builder, so every graph is a valid CSR.  It happens about once per
 * (c + d)^log2(nodes) draws: never in practice at the Graph500 parameters
 * (.57/.19/.19), now and then at the GTGraph defaults (.45/.15/.15).
 */
#pragma once
#include "utils.cuh"

namespace b40c {
namespace graph {
namespace builder {

inline double Drand48() { return double(rand()) / RAND_MAX; }

inline bool Flip() { return rand() >= RAND_MAX / 2; }

template <typename VertexId>
void ChoosePartition(VertexId *u, VertexId *v, VertexId step, double a, double b, double c, double d)
{
    const double p = Drand48();
    // open intervals: a draw landing exactly on a boundary leaves (u, v) unchanged
    if (p < a) {
    } else if (a < p && p < a + b) {
        *v += step;
    } else if (a + b < p && p < a + b + c) {
        *u += step;
    } else if (a + b + c < p && p < a + b + c + d) {
        *u += step;
        *v += step;
    }
}

inline void VaryParams(double *a, double *b, double *c, double *d)
{
    double *q[4] = {a, b, c, d};
    for (int i = 0; i < 4; i++) {
        const bool up = Flip();
        const double delta = *q[i] * 0.05 * Drand48();
        *q[i] = up ? *q[i] + delta : *q[i] - delta;
    }
    const double s = *a + *b + *c + *d;
    *a /= s;
    *b /= s;
    *c /= s;
    *d /= s;
}

template <bool LOAD_VALUES, typename VertexId, typename Value, typename SizeT>
int BuildRmatGraph(SizeT nodes, SizeT edges, CsrGraph<VertexId, Value, SizeT> &csr_graph, bool undirected, double a0,
                   double b0, double c0)
{
    typedef CooEdgeTuple<VertexId, Value> EdgeTupleType;
    if (nodes < 0 || edges < 0) {
        fprintf(stderr, "Invalid graph size: nodes=%lld, edges=%lld", (long long)nodes, (long long)edges);
        return -1;
    }
    printf("  Selecting %llu %s RMAT edges in COO format (a:%f,b:%f,c:%f,d:%f)... ", (unsigned long long)edges,
           undirected ? "undirected" : "directed", a0, b0, c0, 1.0 - (a0 + b0 + c0));
    fflush(stdout);
    time_t t0 = time(NULL);
    const SizeT directed_edges = undirected ? edges * 2 : edges;
    EdgeTupleType *coo = (EdgeTupleType *)malloc(sizeof(EdgeTupleType) * (size_t)(directed_edges > 0 ? directed_edges : 1));
    if (!coo) {
        fprintf(stderr, "BuildRmatGraph: out of memory\n");
        return -1;
    }
    for (SizeT i = 0; i < edges; i++) {
        double a = a0, b = b0, c = c0, d = 1.0 - (a0 + b0 + c0);
        VertexId u = 1, v = 1;
        for (VertexId step = nodes / 2; step >= 1; step /= 2) {
            ChoosePartition(&u, &v, step, a, b, c, d);
            VaryParams(&a, &b, &c, &d);
        }
        if (u == (VertexId)nodes) u = 0;
        if (v == (VertexId)nodes) v = 0;
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
