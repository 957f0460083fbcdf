/*
 * Multi-GPU enactor (drop-in for b40c/graph/bfs/enactor_multi_gpu.cuh:77-914),
 * single-GPU only.  The reference stripes the vertices over several GPUs and
 * exchanges frontiers between them each level; this library searches on one
 * GPU, so the class keeps the reference's interface for callers that name it
 * (its constructor, GetFrontierType, GetStatistics, EnactSearch) and:
 *   - on a problem spread over more than one GPU returns
 *     cudaErrorInvalidConfiguration (CsrProblem::FromHostProblem already
 *     refuses num_gpus != 1, so such a problem cannot be built here);
 *   - on a one-GPU problem runs the expand-contract search, which gives the
 *     labels the reference's multi-GPU enactor computes on one GPU.
 */
#pragma once
#include "../../util/cuda_properties.cuh"
#include "enactor_base.cuh"

namespace b40c {
namespace graph {
namespace bfs {

template <bool INSTRUMENT>
class EnactorMultiGpu : public EnactorBase {
  public:
    EnactorMultiGpu(bool DEBUG = false) : EnactorBase(MULTI_GPU_FRONTIERS, B40C_EXPAND_CONTRACT, INSTRUMENT, DEBUG) {}

    template <typename CsrProblem>
    cudaError_t EnactSearch(CsrProblem &csr_problem, typename CsrProblem::VertexId src, int max_grid_size = 0)
    {
        if (csr_problem.num_gpus > 1)
            return util::B40CPerror(cudaErrorInvalidConfiguration,
                                    "EnactorMultiGpu: this library searches on one GPU", __FILE__, __LINE__);
        return this->Enact(csr_problem, src, B40C_ENACT_FUSED, max_grid_size, (const b40c_bfs_policy *)0);
    }
};

}  // namespace bfs
}  // namespace graph
}  // namespace b40c
