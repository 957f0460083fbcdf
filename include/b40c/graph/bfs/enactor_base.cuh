/*
 * Enactor base (drop-in for b40c/graph/bfs/enactor_base.cuh:55-131): the
 * frontier type of a strategy, DEBUG output, and the common enact path onto
 * the library's b40c_bfs_enact.
 *
 * As in the reference, an Enact*Search call returns once the search's queue
 * overflow status is known (cudaErrorInvalidConfiguration on overflow), so
 * the call synchronises with the device; the statistics are read at the
 * same time.  INSTRUMENT = true turns on per-level records and CTA duty.
 */
#pragma once
#include <stdio.h>

#include "../../util/error_utils.cuh"
#include "b40c_bfs.h"
#include "csr_problem.cuh"

namespace b40c {
namespace graph {
namespace bfs {

class EnactorBase {
  protected:
    FrontierType frontier_type;
    int strategy;
    bool instrument;
    long long total_queued;
    int search_depth;
    double avg_duty;

  public:
    bool DEBUG;

    FrontierType GetFrontierType() { return frontier_type; }

    /* total_queued: sum of the frontier lengths the last search processed;
     * search_depth: its number of levels (max distance + 1); avg_duty: mean
     * busy fraction of the CTAs (INSTRUMENT enactors only, else 0). */
    template <typename VertexId>
    void GetStatistics(long long &total_queued, VertexId &search_depth, double &avg_duty)
    {
        total_queued = this->total_queued;
        search_depth = (VertexId)this->search_depth;
        avg_duty = this->avg_duty;
    }

  protected:
    EnactorBase(FrontierType frontier_type, int strategy, bool instrument, bool DEBUG)
        : frontier_type(frontier_type), strategy(strategy), instrument(instrument), total_queued(0), search_depth(0),
          avg_duty(0.0), DEBUG(DEBUG)
    {
    }

    template <typename CsrProblem>
    cudaError_t Enact(CsrProblem &problem, typename CsrProblem::VertexId src, int mode, int max_grid_size,
                      const b40c_bfs_policy *policy)
    {
        if (!problem.handle)
            return util::B40CPerror(cudaErrorInvalidValue, "enact before FromHostProblem", __FILE__, __LINE__);
        if (instrument) b40c_bfs_set_instrument(problem.handle, 1);
        int rc = b40c_bfs_enact(problem.handle, strategy, mode, (int32_t)src, max_grid_size, policy);
        if (rc) return util::B40CPerror(util::AsCudaError(rc), "BFS enact failed", __FILE__, __LINE__);
        int64_t tq = 0;
        int32_t depth = 0;
        double duty = 0.0;
        rc = b40c_bfs_stats(problem.handle, &tq, &depth, &duty);
        if (rc == B40C_ERROR_INVALID_CONFIGURATION)
            return util::B40CPerror(cudaErrorInvalidConfiguration,
                                    "Frontier queue overflow.  Please increase queue-sizing factor. ", __FILE__,
                                    __LINE__);
        if (rc) return util::B40CPerror(util::AsCudaError(rc), "BFS search failed", __FILE__, __LINE__);
        total_queued = (long long)tq;
        search_depth = depth;
        avg_duty = duty;
        if (DEBUG) {
            printf("DEBUG: strategy %d, src %lld, depth %d, total queued %lld", strategy, (long long)src, depth,
                   (long long)tq);
            if (instrument) printf(", avg duty %.2f%%", duty * 100.0);
            printf("\n");
            fflush(stdout);
        }
        return cudaSuccess;
    }
};

}  // namespace bfs
}  // namespace graph
}  // namespace b40c
