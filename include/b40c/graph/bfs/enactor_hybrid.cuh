/*
 * Hybrid enactor (drop-in for b40c/graph/bfs/enactor_hybrid.cuh:64-758): the fused
 * contract-expand kernel while the edge frontier is small, two-phase level
 * launches while it exceeds gridDim x saturation_quit items.
 */
#pragma once
#include "enactor_base.cuh"

namespace b40c {
namespace graph {
namespace bfs {

template <bool INSTRUMENT>
class EnactorHybrid : public EnactorBase {
  public:
    EnactorHybrid(bool DEBUG = false) : EnactorBase(EDGE_FRONTIERS, B40C_HYBRID, INSTRUMENT, DEBUG) {}

    /* the strategy's default schedule */
    template <typename CsrProblem>
    cudaError_t EnactSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, int max_grid_size = 0)
    {
        return this->Enact(csr_problem, src, B40C_ENACT_FUSED, max_grid_size, (const b40c_bfs_policy *)0);
    }

    /* same, with an explicit runtime kernel policy (in place of the reference's
     * compile-time KernelPolicy template argument) */
    template <typename CsrProblem>
    cudaError_t EnactSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, const b40c_bfs_policy &policy,
                        int max_grid_size = 0)
    {
        return this->Enact(csr_problem, src, B40C_ENACT_FUSED, max_grid_size, &policy);
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
