// Launch helpers shared by the enactor translation units.
#pragma once
#include "bfs_kernels.cuh"
#include "problem.h"

namespace b40c {
namespace rt {

// Dynamic shared memory of the vertex/edge kernels: their state, plus the
// history cull table and the bottom-up prefetch buffer when the policy turns
// them on, plus the warp-autonomous levels' tables for CTAs of more than 256
// threads (smaller CTAs keep them in their sub-round arrays); the same order
// as hist_init.
template <typename Smem>
inline size_t kernel_smem(const b40c_bfs_policy &pol)
{
    return ((sizeof(Smem) + 15) & ~size_t(15)) + (pol.history_cull > 0 ? sizeof(uint32_t) << kHistLog : 0) +
           (pol.bottom_up_prefetch > 0 ? dev::kBuPrefetchBytes : 0) +
           (pol.warp_contract > 0 && pol.threads > 256 ? (size_t)(pol.threads / 32) * dev::kWarpTableBytes : 0);
}

// Grid of the set-up kernel: the full label/mask initialisation is a
// grid-stride fill, the source-only set-up a single CTA.
inline int init_grid(b40c_bfs_problem *p, bool full)
{
    return full ? std::max(1, std::min<int>(p->sms * 8, (int)((p->nodes + kThreads - 1) / kThreads))) : 1;
}

template <bool PRED>
const void *init_kernel_ptr(bool vertex_frontier, bool full)
{
    if (vertex_frontier)
        return full ? (const void *)dev::init_kernel<PRED, true, true> : (const void *)dev::init_kernel<PRED, true, false>;
    return full ? (const void *)dev::init_kernel<PRED, false, true> : (const void *)dev::init_kernel<PRED, false, false>;
}

template <bool PRED>
int launch_init(b40c_bfs_problem *p, const BfsParams &k, bool vertex_frontier, bool full)
{
    BfsParams kk = k;
    void *args[] = {&kk};
    CUDA_TRY(cudaLaunchKernel(init_kernel_ptr<PRED>(vertex_frontier, full), dim3(init_grid(p, full)), dim3(kThreads),
                              args, 0, p->stream),
             "init kernel launch");
    return B40C_SUCCESS;
}

// Common start of an enact: stores (source, depth limit) in this enact's
// pinned ring slot and records the enact's start event.  The slot was last
// used kRing enacts ago; its search (and so its upload) must have finished
// before the pair is overwritten.
inline int begin_enact(b40c_bfs_problem *p, int32_t src, int32_t depth_limit)
{
    const int slot = p->ring_pos;
    if (p->ring_count == b40c_bfs_problem::kRing)
        CUDA_TRY(cudaEventSynchronize(p->ring_b[slot]), "source slot reuse wait");
    p->h_src_ring[2 * slot] = src;
    p->h_src_ring[2 * slot + 1] = depth_limit;
    CUDA_TRY(cudaEventRecord(p->ev0, p->stream), "event record");
    return B40C_SUCCESS;
}

inline int upload_source(b40c_bfs_problem *p)
{
    CUDA_TRY(cudaMemcpyAsync(&p->st->src, source_slot(p), 2 * sizeof(int32_t), cudaMemcpyHostToDevice, p->stream),
             "source upload");
    return B40C_SUCCESS;
}

inline int mark_search_start(b40c_bfs_problem *p)
{
    CUDA_TRY(cudaEventRecord(p->ring_a[p->ring_pos], p->stream), "event record");
    return B40C_SUCCESS;
}

inline int launch_cooperative(b40c_bfs_problem *p, const void *kern, int grid, int block, size_t smem, BfsParams &k,
                              const char *what)
{
    void *args[] = {&k};
    CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(block), args, smem, p->stream), what);
    return B40C_SUCCESS;
}

inline int launch_plain(b40c_bfs_problem *p, const void *kern, int grid, int block, size_t smem, BfsParams &k,
                        const char *what)
{
    void *args[] = {&k};
    CUDA_TRY(cudaLaunchKernel(kern, dim3(grid), dim3(block), args, smem, p->stream), what);
    return B40C_SUCCESS;
}

// Kernel variants are built for these CTA sizes (policy.threads).
constexpr int kCtaSizes[3] = {128, 256, 512};

// Test-only fault injection: B40C_TEST_SKIP_ARRIVAL_CTA=<cta> makes that CTA
// of a persistent launch leave at its first whole-grid end-of-level barrier
// without arriving (and without reporting anything), so the other CTAs'
// bounded waits must run out; the search then reports
// B40C_ERROR_LAUNCH_TIMEOUT.  B40C_TEST_SPIN_LIMIT (make_params) shortens
// those waits.
inline int injected_skip_cta()
{
    const char *inj = getenv("B40C_TEST_SKIP_ARRIVAL_CTA");
    return inj ? atoi(inj) : -1;
}

// Test-only: B40C_TEST_LATE_START_NS=<ns> (at most 10 ms) makes every CTA
// but CTA 0 of a persistent launch start that much later, as a CTA the
// hardware schedules late would: the first levels then run while most of
// the grid has not read its start state yet.
inline uint32_t injected_late_start_ns()
{
    const char *inj = getenv("B40C_TEST_LATE_START_NS");
    const long v = inj ? atol(inj) : 0;
    return v > 0 ? (uint32_t)std::min(v, 10000000L) : 0u;
}

}  // namespace rt
}  // namespace b40c
