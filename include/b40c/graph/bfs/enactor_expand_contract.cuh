/*
 * Expand-contract enactor (drop-in for b40c/graph/bfs/enactor_expand_contract.cuh:59-526):
 * vertex frontiers; each level expands the frontier's adjacency lists and
 * culls every neighbour on the spot (edge-balanced per-CTA ranges).
 * Unlike the reference, predecessor marking is supported.
 */
#pragma once
#include "enactor_base.cuh"

namespace b40c {
namespace graph {
namespace bfs {

template <bool INSTRUMENT>
class EnactorExpandContract : public EnactorBase {
  public:
    EnactorExpandContract(bool DEBUG = false) : EnactorBase(VERTEX_FRONTIERS, B40C_EXPAND_CONTRACT, INSTRUMENT, DEBUG) {}

    /* one persistent grid, bounded software barrier between levels */
    template <typename CsrProblem>
    cudaError_t EnactFusedSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, int max_grid_size = 0)
    {
        return this->Enact(csr_problem, src, B40C_ENACT_FUSED, max_grid_size, (const b40c_bfs_policy *)0);
    }

    /* same, with an explicit runtime kernel policy (in place of the reference's
     * compile-time KernelPolicy template argument) */
    template <typename CsrProblem>
    cudaError_t EnactFusedSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, const b40c_bfs_policy &policy,
                        int max_grid_size = 0)
    {
        return this->Enact(csr_problem, src, B40C_ENACT_FUSED, max_grid_size, &policy);
    }

    /* one launch (or phase pair) per level */
    template <typename CsrProblem>
    cudaError_t EnactIterativeSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, int max_grid_size = 0)
    {
        return this->Enact(csr_problem, src, B40C_ENACT_ITERATIVE, max_grid_size, (const b40c_bfs_policy *)0);
    }

    /* same, with an explicit runtime kernel policy (in place of the reference's
     * compile-time KernelPolicy template argument) */
    template <typename CsrProblem>
    cudaError_t EnactIterativeSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, const b40c_bfs_policy &policy,
                        int max_grid_size = 0)
    {
        return this->Enact(csr_problem, src, B40C_ENACT_ITERATIVE, max_grid_size, &policy);
    }

    /* the whole search replayed as one CUDA graph */
    template <typename CsrProblem>
    cudaError_t EnactGraphSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, int max_grid_size = 0)
    {
        return this->Enact(csr_problem, src, B40C_ENACT_GRAPH, max_grid_size, (const b40c_bfs_policy *)0);
    }

    /* same, with an explicit runtime kernel policy (in place of the reference's
     * compile-time KernelPolicy template argument) */
    template <typename CsrProblem>
    cudaError_t EnactGraphSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, const b40c_bfs_policy &policy,
                        int max_grid_size = 0)
    {
        return this->Enact(csr_problem, src, B40C_ENACT_GRAPH, max_grid_size, &policy);
    }
};

}  // namespace bfs
}  // namespace graph
}  // namespace b40c
