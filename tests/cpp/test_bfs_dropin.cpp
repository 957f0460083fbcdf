// A caller of the reference's C++ BFS API, unchanged apart from the include
// path: builds a graph with the b40c builders, searches it with each
// enactor the way the reference's test driver does (fused contract-expand
// and expand-contract, iterative two-phase, hybrid EnactSearch) and checks
// the labels against a serial CPU BFS.  Exit status 0 iff every search
// validates.
//
//   test_bfs_dropin <grid2d W | grid3d W | rmat N M | random N M | rr N D>
//                   [--mark-pred] [--src=S] [--queue-sizing=Q] [--instrumented]
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <deque>
#include <string>
#include <vector>

#include <b40c/graph/builder/grid2d.cuh>
#include <b40c/graph/builder/grid3d.cuh>
#include <b40c/graph/builder/random.cuh>
#include <b40c/graph/builder/rmat.cuh>
#include <b40c/graph/builder/rr.cuh>
#include <b40c/graph/bfs/csr_problem.cuh>
#include <b40c/graph/bfs/enactor_contract_expand.cuh>
#include <b40c/graph/bfs/enactor_direction_optimizing.cuh>
#include <b40c/graph/bfs/enactor_expand_contract.cuh>
#include <b40c/graph/bfs/enactor_hybrid.cuh>
#include <b40c/graph/bfs/enactor_two_phase.cuh>

using namespace b40c;
using namespace b40c::graph;

typedef int VertexId;
typedef int Value;
typedef int SizeT;

static void CpuBfs(const CsrGraph<VertexId, Value, SizeT> &g, VertexId src, std::vector<VertexId> &dist)
{
    dist.assign(g.nodes, -1);
    std::deque<VertexId> q;
    dist[src] = 0;
    q.push_back(src);
    while (!q.empty()) {
        VertexId u = q.front();
        q.pop_front();
        for (SizeT e = g.row_offsets[u]; e < g.row_offsets[u + 1]; e++) {
            VertexId v = g.column_indices[e];
            if (dist[v] < 0) {
                dist[v] = dist[u] + 1;
                q.push_back(v);
            }
        }
    }
}

static bool Validate(const CsrGraph<VertexId, Value, SizeT> &g, bool mark_pred, const std::vector<VertexId> &dist,
                     const std::vector<VertexId> &labels)
{
    for (SizeT v = 0; v < g.nodes; v++) {
        if (!mark_pred) {
            if (labels[v] != dist[v]) {
                printf("INCORRECT: vertex %d label %d, expected %d\n", v, labels[v], dist[v]);
                return false;
            }
            continue;
        }
        VertexId parent = labels[v];
        if (parent < 0) {
            if (dist[v] > 0) {
                printf("INCORRECT: reached vertex %d has no parent\n", v);
                return false;
            }
            continue;
        }
        bool adjacent = false;
        for (SizeT e = g.row_offsets[parent]; e < g.row_offsets[parent + 1]; e++) adjacent |= g.column_indices[e] == v;
        if (dist[parent] + 1 != dist[v] || !adjacent) {
            printf("INCORRECT: parent %d of vertex %d\n", parent, v);
            return false;
        }
    }
    return true;
}

template <bool MARK_PRED, typename Enactor, typename EnactFn>
static bool RunOne(const char *name, Enactor &enactor, EnactFn enact, bfs::CsrProblem<VertexId, SizeT, MARK_PRED> &problem,
                   const CsrGraph<VertexId, Value, SizeT> &g, double queue_sizing, const std::vector<VertexId> &dist)
{
    if (problem.Reset(enactor.GetFrontierType(), queue_sizing)) return false;
    if (enact()) return false;
    long long total_queued = 0;
    VertexId depth = 0;
    double duty = 0;
    enactor.GetStatistics(total_queued, depth, duty);
    std::vector<VertexId> labels(g.nodes);
    if (problem.ExtractResults(labels.data())) return false;
    bool ok = Validate(g, MARK_PRED, dist, labels);
    printf("[%s] %s  depth %d  total queued %lld  duty %.2f\n", name, ok ? "CORRECT" : "INCORRECT", (int)depth,
           total_queued, duty);
    return ok;
}

template <bool MARK_PRED>
static int Run(CsrGraph<VertexId, Value, SizeT> &g, VertexId src, double queue_sizing, bool instrumented)
{
    bfs::CsrProblem<VertexId, SizeT, MARK_PRED> problem;
    if (problem.FromHostProblem(false, g.nodes, g.edges, g.column_indices, g.row_offsets, 1)) return 1;
    std::vector<VertexId> dist;
    CpuBfs(g, src, dist);
    bool ok = true;
    bfs::EnactorExpandContract<false> expand_contract;
    bfs::EnactorContractExpand<false> contract_expand;
    bfs::EnactorTwoPhase<false> two_phase;
    bfs::EnactorHybrid<false> hybrid;
    bfs::EnactorDirectionOptimizing<false> direction_optimizing;
    // the reference driver's choices: fused CE and EC, iterative two-phase, hybrid EnactSearch
    ok &= RunOne("expand-contract", expand_contract, [&] { return expand_contract.EnactFusedSearch(problem, src); },
                 problem, g, queue_sizing, dist);
    ok &= RunOne("contract-expand", contract_expand, [&] { return contract_expand.EnactFusedSearch(problem, src); },
                 problem, g, queue_sizing, dist);
    ok &= RunOne("two-phase", two_phase, [&] { return two_phase.EnactIterativeSearch(problem, src); }, problem, g,
                 queue_sizing, dist);
    ok &= RunOne("hybrid", hybrid, [&] { return hybrid.EnactSearch(problem, src); }, problem, g, queue_sizing, dist);
    ok &= RunOne("direction-optimizing", direction_optimizing,
                 [&] { return direction_optimizing.EnactSearch(problem, src); }, problem, g, queue_sizing, dist);
    ok &= RunOne("expand-contract (graph)", expand_contract,
                 [&] { return expand_contract.EnactGraphSearch(problem, src); }, problem, g, queue_sizing, dist);
    if (instrumented) {
        bfs::EnactorExpandContract<true> instrumented_ec(true);
        ok &= RunOne("expand-contract (instrumented)", instrumented_ec,
                     [&] { return instrumented_ec.EnactIterativeSearch(problem, src); }, problem, g, queue_sizing,
                     dist);
    }
    return ok ? 0 : 1;
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s <grid2d W | grid3d W | rmat N M | random N M | rr N D> [flags]\n", argv[0]);
        return 2;
    }
    srand(0);
    std::string type = argv[1];
    bool mark_pred = false, instrumented = false;
    long long src = -1;
    double queue_sizing = 1.3;
    for (int i = 2; i < argc; i++) {
        if (!strcmp(argv[i], "--mark-pred")) mark_pred = true;
        if (!strcmp(argv[i], "--instrumented")) instrumented = true;
        if (!strncmp(argv[i], "--src=", 6)) src = atoll(argv[i] + 6);
        if (!strncmp(argv[i], "--queue-sizing=", 15)) queue_sizing = atof(argv[i] + 15);
    }
    CsrGraph<VertexId, Value, SizeT> g;
    int rc = -1;
    if (type == "grid2d") rc = builder::BuildGrid2dGraph<false>((VertexId)atoi(argv[2]), g);
    else if (type == "grid3d") rc = builder::BuildGrid3dGraph<false>((VertexId)atoi(argv[2]), g);
    else if (type == "rmat" && argc > 3) rc = builder::BuildRmatGraph<false>((SizeT)atoi(argv[2]), (SizeT)atoi(argv[3]), g, true, 0.57, 0.19, 0.19);
    else if (type == "random" && argc > 3) rc = builder::BuildRandomGraph<false>((SizeT)atoi(argv[2]), (SizeT)atoi(argv[3]), g, true);
    else if (type == "rr" && argc > 3) rc = builder::BuildRandomRegularishGraph<false>((SizeT)atoi(argv[2]), atoi(argv[3]), g);
    if (rc != 0) {
        fprintf(stderr, "graph construction failed\n");
        return 2;
    }
    g.PrintHistogram();
    if (src < 0) {
        // first vertex with an edge
        for (src = 0; src < g.nodes && g.row_offsets[src + 1] == g.row_offsets[src]; src++) {}
    }
    return mark_pred ? Run<true>(g, (VertexId)src, queue_sizing, instrumented)
                     : Run<false>(g, (VertexId)src, queue_sizing, instrumented);
}
