// Harness that exposes the reference's own host code through a C ABI so the
// oracle and the builders can be checked against it.  TEST INFRASTRUCTURE ONLY.
//
// It is compiled by oracle/build_ref.sh against the reference tree (include
// path) into oracle/_ref/libb40c_ref.so; nothing of the reference is copied
// into this repository.  The reference's SimpleReferenceBfs lives inside its
// driver test/bfs/test_bfs.cu:503-578, which also includes every GPU kernel
// and therefore does not compile with CUDA 12; build_ref.sh extracts just that
// function's text into oracle/_ref/ and this file supplies the few driver
// helpers it calls (Stats, DisplayStats, Histogram, g_verbose).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <deque>

#include <b40c_test_util.h>
#include <b40c/graph/builder/utils.cuh>
#include <b40c/graph/coo_edge_tuple.cuh>
#include <b40c/graph/csr_graph.cuh>
#include <b40c/graph/builder/grid2d.cuh>
#include <b40c/graph/builder/grid3d.cuh>
#include <b40c/graph/builder/rmat.cuh>
#include <b40c/graph/builder/random.cuh>
#include <b40c/graph/builder/rr.cuh>
#include <sstream>
#include <vector>
#include <b40c/graph/builder/market.cuh>
#include <b40c/graph/builder/dimacs.cuh>
#include <b40c/graph/builder/metis.cuh>

using namespace b40c;
using namespace b40c::graph;

// ---- helpers the extracted driver function refers to ----------------------
static bool g_verbose = false;

struct Stats {
    const char *name;
    Stats() : name("ref") {}
};

static long long g_last_search_depth = 0;
static double g_last_elapsed_ms = 0.0;

template <bool MARK_PREDECESSORS, typename VertexId, typename Value, typename SizeT>
void DisplayStats(Stats &, VertexId, VertexId *, VertexId *,
                  const CsrGraph<VertexId, Value, SizeT> &, double elapsed,
                  VertexId search_depth, long long, double)
{
    g_last_search_depth = search_depth;
    g_last_elapsed_ms = elapsed;
}

template <typename VertexId, typename Value, typename SizeT>
void Histogram(VertexId, VertexId *, const CsrGraph<VertexId, Value, SizeT> &, VertexId) {}

#include "_ref/simple_reference_bfs.inc"

// ---- C ABI ------------------------------------------------------------------
typedef CsrGraph<int, int, int> Graph;

// Runs the reference SimpleReferenceBfs on caller-owned CSR arrays.
extern "C" int ref_simple_bfs(int32_t nodes, int32_t edges, int32_t *row_offsets,
                              int32_t *column_indices, int32_t src, int32_t *labels,
                              int64_t *search_depth, double *elapsed_user_ms)
{
    Graph g;
    g.nodes = nodes;
    g.edges = edges;
    g.row_offsets = row_offsets;
    g.column_indices = column_indices;
    Stats stats;
    SimpleReferenceBfs(0, g, labels, src, stats);
    // the graph does not own the caller's arrays
    g.row_offsets = NULL;
    g.column_indices = NULL;
    g.nodes = g.edges = 0;
    *search_depth = g_last_search_depth;
    *elapsed_user_ms = g_last_elapsed_ms;
    return 0;
}

static int take(Graph &g, int32_t **ro, int32_t **ci, int64_t *n, int64_t *m)
{
    *ro = g.row_offsets;
    *ci = g.column_indices;
    *n = g.nodes;
    *m = g.edges;
    g.row_offsets = NULL;
    g.column_indices = NULL;
    g.nodes = g.edges = 0;
    return 0;
}

extern "C" int ref_build_grid2d(int32_t width, int32_t **ro, int32_t **ci, int64_t *n, int64_t *m)
{
    Graph g;
    if (builder::BuildGrid2dGraph<false>(width, g) != 0) return -1;
    return take(g, ro, ci, n, m);
}

extern "C" int ref_build_grid3d(int32_t width, int32_t **ro, int32_t **ci, int64_t *n, int64_t *m)
{
    Graph g;
    if (builder::BuildGrid3dGraph<false>(width, g) != 0) return -1;
    return take(g, ro, ci, n, m);
}

extern "C" int ref_build_rmat(int32_t nodes, int32_t edges, int undirected, double a, double b,
                              double c, unsigned seed, int32_t **ro, int32_t **ci, int64_t *n,
                              int64_t *m)
{
    Graph g;
    srand(seed);
    if (builder::BuildRmatGraph<false>(nodes, edges, g, undirected != 0, a, b, c) != 0) return -1;
    return take(g, ro, ci, n, m);
}

extern "C" int ref_build_random(int32_t nodes, int32_t edges, int undirected, unsigned seed,
                                int32_t **ro, int32_t **ci, int64_t *n, int64_t *m)
{
    Graph g;
    srand(seed);
    if (builder::BuildRandomGraph<false>(nodes, edges, g, undirected != 0) != 0) return -1;
    return take(g, ro, ci, n, m);
}

extern "C" int ref_build_rr(int32_t nodes, int32_t degree, unsigned seed, int32_t **ro,
                            int32_t **ci, int64_t *n, int64_t *m)
{
    Graph g;
    srand(seed);
    if (builder::BuildRandomRegularishGraph<false>(nodes, degree, g) != 0) return -1;
    return take(g, ro, ci, n, m);
}

extern "C" int32_t ref_random_node(int32_t nodes, unsigned seed, int reseed)
{
    if (reseed) srand(seed);
    return builder::RandomNode(nodes);
}

// The reference's graph file readers (market.cuh, dimacs.cuh, metis.cuh).
extern "C" int ref_read_market(const char *path, int undirected, int32_t **ro, int32_t **ci, int64_t *n,
                               int64_t *m)
{
    Graph g;
    if (builder::BuildMarketGraph<false>((char *)path, g, undirected != 0) != 0) return -1;
    return take(g, ro, ci, n, m);
}

extern "C" int ref_read_dimacs(const char *path, int undirected, int splice, int32_t **ro, int32_t **ci,
                               int64_t *n, int64_t *m)
{
    Graph g;
    if (builder::BuildDimacsGraph<false>((char *)path, g, undirected != 0, splice) != 0) return -1;
    return take(g, ro, ci, n, m);
}

extern "C" int ref_read_metis(const char *path, int32_t **ro, int32_t **ci, int64_t *n, int64_t *m)
{
    Graph g;
    if (builder::BuildMetisGraph<false>((char *)path, g) != 0) return -1;
    return take(g, ro, ci, n, m);
}

extern "C" void ref_free(void *p) { free(p); }
