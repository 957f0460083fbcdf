/*
 * Host CSR graph (drop-in for b40c/graph/csr_graph.cuh:51-245).
 *
 * Same members (nodes, edges, row_offsets, column_indices, values, pinned)
 * and methods (FromScratch, FromCoo, PrintHistogram, DisplayGraph, Free).
 * Pinned graphs use mapped page-locked memory from the library
 * (b40c_host_alloc), so a CsrProblem can stream them from the host.
 */
#pragma once
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include <algorithm>

#include "../util/basic_utils.cuh"
#include "../util/error_utils.cuh"
#include "b40c_bfs.h"
#include "coo_edge_tuple.cuh"

namespace b40c {
namespace graph {

template <typename VertexId, typename Value, typename SizeT>
struct CsrGraph {
    SizeT nodes;
    SizeT edges;

    SizeT *row_offsets;
    VertexId *column_indices;
    Value *values;

    bool pinned;

    CsrGraph(bool pinned = false) : nodes(0), edges(0), row_offsets(NULL), column_indices(NULL), values(NULL),
                                    pinned(pinned)
    {
    }

    /* Allocates storage for `nodes` vertices and `edges` edges (csr_graph.cuh:76-102);
     * exits on an allocation failure like the reference. */
    template <bool LOAD_VALUES>
    void FromScratch(SizeT nodes, SizeT edges)
    {
        Free();
        this->nodes = nodes;
        this->edges = edges;
        row_offsets = (SizeT *)Allocate(sizeof(SizeT) * (size_t)(nodes + 1), "row_offsets");
        column_indices = (VertexId *)Allocate(sizeof(VertexId) * (size_t)(edges > 0 ? edges : 1), "column_indices");
        values = LOAD_VALUES ? (Value *)Allocate(sizeof(Value) * (size_t)(edges > 0 ? edges : 1), "values") : NULL;
    }

    /* CSR of a COO edge list (csr_graph.cuh:109-152): stable sort by row (so each
     * row keeps the list's order), then row offsets with empty rows filled in. */
    template <bool LOAD_VALUES, typename Tuple>
    void FromCoo(Tuple *coo, SizeT coo_nodes, SizeT coo_edges, bool ordered_rows = false)
    {
        printf("  Converting %lld vertices, %lld directed edges (%s tuples) to CSR format... ", (long long)coo_nodes,
               (long long)coo_edges, ordered_rows ? "ordered" : "unordered");
        time_t t0 = time(NULL);
        fflush(stdout);
        FromScratch<LOAD_VALUES>(coo_nodes, coo_edges);
        if (!ordered_rows) std::stable_sort(coo, coo + coo_edges, DimacsTupleCompare<Tuple>);
        SizeT e = 0;
        for (SizeT row = 0; row <= nodes; row++) {
            row_offsets[row] = e;
            while (e < coo_edges && (SizeT)coo[e].row == row) {
                column_indices[e] = coo[e].col;
                if (LOAD_VALUES) coo[e].Val(values[e]);
                e++;
            }
        }
        // rows past the last vertex id (a builder's out-of-range id) stay after row_offsets[nodes]
        for (; e < coo_edges; e++) {
            column_indices[e] = coo[e].col;
            if (LOAD_VALUES) coo[e].Val(values[e]);
        }
        printf("Done converting (%ds).\n", (int)(time(NULL) - t0));
        fflush(stdout);
    }

    /* Log2 degree histogram (csr_graph.cuh:157-190). */
    void PrintHistogram()
    {
        fflush(stdout);
        long long counts[34] = {0};
        int top = -1;
        for (SizeT v = 0; v < nodes; v++) {
            long long d = (long long)(row_offsets[v + 1] - row_offsets[v]);
            int lg = -1;
            while (d > 0) {
                d >>= 1;
                lg++;
            }
            if (lg > top) top = lg;
            counts[lg + 1]++;
        }
        printf("\nDegree Histogram (%lld vertices, %lld directed edges):\n", (long long)nodes, (long long)edges);
        for (int i = -1; i < top + 1; i++)
            printf("\tDegree 2^%i: %lld (%.2f%%)\n", i, counts[i + 1], nodes ? counts[i + 1] * 100.0 / nodes : 0.0);
        printf("\n");
        fflush(stdout);
    }

    void DisplayGraph()
    {
        printf("Input Graph:\n");
        for (SizeT v = 0; v < nodes; v++) {
            PrintValue(v);
            printf(": ");
            for (SizeT e = row_offsets[v]; e < row_offsets[v + 1]; e++) {
                PrintValue(column_indices[e]);
                printf(", ");
            }
            printf("\n");
        }
    }

    void Free()
    {
        Release(row_offsets);
        Release(column_indices);
        Release(values);
        row_offsets = NULL;
        column_indices = NULL;
        values = NULL;
        nodes = 0;
        edges = 0;
    }

    ~CsrGraph() { Free(); }

  private:
    void *Allocate(size_t bytes, const char *what)
    {
        void *p = NULL;
        if (pinned) {
            if (util::B40CPerror(util::AsCudaError(b40c_host_alloc(&p, bytes, 1)), "CsrGraph pinned allocation failed",
                                 __FILE__, __LINE__)) {
                fprintf(stderr, "(%s)\n", what);
                exit(1);
            }
        } else {
            p = malloc(bytes);
            if (!p) {
                fprintf(stderr, "CsrGraph: malloc of %s failed\n", what);
                exit(1);
            }
        }
        return p;
    }
    void Release(void *p)
    {
        if (!p) return;
        if (pinned)
            b40c_host_free(p);
        else
            free(p);
    }
    CsrGraph(const CsrGraph &);
    CsrGraph &operator=(const CsrGraph &);
};

}  // namespace graph
}  // namespace b40c
