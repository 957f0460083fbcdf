// Batched multi-source BFS: up to 64 sources per launch, per-source depth
// limits, labels kept on the device as [k][n] (source-major).
#include <algorithm>
#include <utility>
#include <vector>

#include "launch_common.cuh"
#include "msbfs_kernels.cuh"

namespace b40c {
namespace rt {

constexpr int kBatchPullAlpha = 6;

void free_batch(b40c_bfs_problem *p)
{
    if (p->d_ms_visited) cudaFree(p->d_ms_visited);
    for (int i = 0; i < 2; i++)
        if (p->d_ms_fmask[i]) cudaFree(p->d_ms_fmask[i]);
    if (p->d_ms_labels) cudaFree(p->d_ms_labels);
    if (p->d_ms_src) cudaFree(p->d_ms_src);
    if (p->d_ms_depth) cudaFree(p->d_ms_depth);
    p->d_ms_visited = nullptr;
    p->d_ms_fmask[0] = p->d_ms_fmask[1] = nullptr;
    p->d_ms_labels = nullptr;
    p->d_ms_src = nullptr;
    p->d_ms_depth = nullptr;
    p->ms_labels_k = 0;
}

int ensure_batch(b40c_bfs_problem *p, int k)
{
    int rc;
    const size_t n = (size_t)p->nodes;
    if (!p->d_ms_visited) {
        if ((rc = alloc_dev((void **)&p->d_ms_visited, sizeof(unsigned long long) * n, "batch visited masks"))) return rc;
        for (int i = 0; i < 2; i++)
            if ((rc = alloc_dev((void **)&p->d_ms_fmask[i], sizeof(unsigned long long) * n, "batch frontier masks")))
                return rc;
        if ((rc = alloc_dev((void **)&p->d_ms_src, sizeof(int32_t) * 64, "batch depth limits"))) return rc;
        if ((rc = alloc_dev((void **)&p->d_ms_depth, sizeof(int32_t) * 64, "batch search depths"))) return rc;
    }
    if (p->ms_labels_k < k) {
        if (p->d_ms_labels) cudaFree(p->d_ms_labels);
        p->d_ms_labels = nullptr;
        p->ms_labels_k = 0;
        if ((rc = alloc_dev((void **)&p->d_ms_labels, sizeof(int32_t) * n * (size_t)k, "batch labels"))) return rc;
        p->ms_labels_k = k;
    }
    return B40C_SUCCESS;
}

int enact_batch(b40c_bfs_problem *p, const int32_t *sources, const int32_t *limits, int k, int max_grid,
                const b40c_bfs_policy &pol)
{
    int rc;
    if ((rc = ensure_vf(p, 0, cap_of(p->queue_sizing, p->nodes)))) return rc;
    if ((rc = ensure_vf(p, 1, cap_of(p->queue_sizing, p->nodes)))) return rc;
    if ((rc = ensure_slots(p))) return rc;
    if ((rc = ensure_batch(p, k))) return rc;
    if ((rc = check_symmetric(p))) return rc;
    if (p->symmetric == 1 && pol.bottom_up_hub_probes > 0 && (rc = ensure_hubs(p))) return rc;
    // distinct source vertices with their combined source masks; they travel
    // to the device as kernel arguments, so nothing on the host is reused
    // while an earlier batch is still queued
    std::vector<std::pair<int32_t, unsigned long long>> ds;
    for (int s = 0; s < k; s++) ds.push_back({sources[s], 1ull << s});
    std::sort(ds.begin(), ds.end());
    int nd = 0;
    for (size_t i = 0; i < ds.size(); i++) {
        if (nd > 0 && ds[nd - 1].first == ds[i].first)
            ds[nd - 1].second |= ds[i].second;
        else
            ds[nd++] = ds[i];
    }
    dev::MsSeed seed{};
    for (int i = 0; i < nd; i++) {
        seed.src[i] = ds[i].first;
        seed.mask[i] = ds[i].second;
    }
    for (int s = 0; s < k; s++) seed.limit[s] = limits ? limits[s] : -1;
    seed.n_distinct = nd;

    BfsParams bp = make_params(p, pol);
    if (p->symmetric != 1) bp.hub2 = nullptr;  // pull levels (and so the pair) only on symmetric graphs
    dev::MsParams m{};
    m.visited = p->d_ms_visited;
    m.fmask[0] = p->d_ms_fmask[0];
    m.fmask[1] = p->d_ms_fmask[1];
    m.labels = p->d_ms_labels;
    m.depth_limit = p->d_ms_src;
    m.depth = p->d_ms_depth;
    m.k = k;
    m.pull_ok = p->symmetric == 1 ? 1 : 0;
    const void *kern = (const void *)dev::msbfs_kernel<kThreads>;
    const size_t smem = sizeof(dev::MsSmem<kThreads>);
    int grid = 0;
    if ((rc = persistent_grid(p, kern, pol, max_grid, smem, &grid))) return rc;
    CUDA_TRY(cudaEventRecord(p->ev0, p->stream), "event record");
    if ((rc = begin_instrumented(p))) return rc;
    const int init_blocks = std::max(1, std::min<int>(p->sms * 8, (int)(((long long)p->nodes + 255) / 256)));
    dev::msbfs_init_kernel<<<init_blocks, kThreads, 0, p->stream>>>(bp, m);
    CUDA_TRY(cudaGetLastError(), "batch init launch");
    dev::msbfs_seed_kernel<<<1, 32, 0, p->stream>>>(bp, m, p->d_ms_src, seed);
    CUDA_TRY(cudaGetLastError(), "batch seed launch");
    if ((rc = mark_search_start(p))) return rc;
    void *args[] = {&bp, &m};
    CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kThreads), args, smem, p->stream),
             "cooperative launch of the batched kernel");
    p->ms_k = k;
    p->needs_init = true;  // the single-source labels/mask are untouched but the queues were reused
    return finish_timing(p);
}

}  // namespace rt
}  // namespace b40c

using namespace b40c;
using namespace b40c::rt;

extern "C" {

int b40c_msbfs_enact(b40c_bfs_problem *p, const int32_t *sources, const int32_t *depth_limits, int k, int max_grid_size,
                     const b40c_bfs_policy *policy)
{
    b40c::clear_error();
    if (!p || !sources || k < 1 || k > 64) return b40c::fail(B40C_ERROR_INVALID_VALUE, "a batch needs 1..64 sources");
    for (int s = 0; s < k; s++)
        if (sources[s] < 0 || sources[s] >= p->nodes)
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "batch source %d (= %d) out of range", s, sources[s]);
    if (max_grid_size < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "negative max_grid_size");
    b40c_bfs_policy pol;
    int rc = resolve_policy(B40C_EXPAND_CONTRACT, policy, &pol);
    if (rc) return rc;
    // batches pull once a level's frontier holds more than 1/6 of the edges
    // (measured on B200: R-MAT 20 batches 4.46 ms at 1/14, 0.82 ms at 1/6;
    // lattices and uniform graphs unchanged or slightly faster)
    if (!policy || policy->bottom_up_alpha == 0) pol.bottom_up_alpha = kBatchPullAlpha;
    DeviceGuard guard(p->device);
    return enact_batch(p, sources, depth_limits, k, max_grid_size, pol);
}

int b40c_msbfs_extract(b40c_bfs_problem *p, int slot, int32_t *h_labels)
{
    b40c::clear_error();
    if (!p || !h_labels) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    if (slot < 0 || slot >= p->ms_k) return b40c::fail(B40C_ERROR_INVALID_VALUE, "no source %d in the last batch", slot);
    DeviceGuard guard(p->device);
    int rc = read_state(p);
    if (rc) return rc;
    if ((rc = check_state_errors(p))) return rc;
    CUDA_TRY(cudaMemcpyAsync(h_labels, p->d_ms_labels + (size_t)slot * (size_t)p->nodes, sizeof(int32_t) * p->nodes,
                             cudaMemcpyDeviceToHost, p->stream),
             "batch label copy");
    CUDA_TRY(cudaStreamSynchronize(p->stream), "batch label copy synchronize");
    return B40C_SUCCESS;
}

int b40c_msbfs_stats(b40c_bfs_problem *p, int32_t *search_depths)
{
    b40c::clear_error();
    if (!p || !search_depths) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    if (p->ms_k < 1) return b40c::fail(B40C_ERROR_NOT_READY, "no batch has run");
    DeviceGuard guard(p->device);
    int rc = read_state(p);
    if (rc) return rc;
    if ((rc = check_state_errors(p))) return rc;
    CUDA_TRY(cudaMemcpyAsync(search_depths, p->d_ms_depth, sizeof(int32_t) * p->ms_k, cudaMemcpyDeviceToHost,
                             p->stream),
             "batch depth copy");
    CUDA_TRY(cudaStreamSynchronize(p->stream), "batch depth copy synchronize");
    return B40C_SUCCESS;
}

int b40c_msbfs_device_labels(b40c_bfs_problem *p, void **d_labels, int32_t *k)
{
    b40c::clear_error();
    if (!p || !d_labels || !k) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    *d_labels = p->d_ms_labels;
    *k = p->ms_k;
    return B40C_SUCCESS;
}

}  // extern "C"
