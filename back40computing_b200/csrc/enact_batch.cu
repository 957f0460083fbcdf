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
    if (p->d_ms_off) cudaFree(p->d_ms_off);
    if (p->join_stream) cudaStreamSynchronize(p->join_stream);
    if (p->d_ms_join) cudaFree(p->d_ms_join);
    if (p->h_ms_join) cudaFreeHost(p->h_ms_join);
    if (p->h_ms_seq) cudaFreeHost(p->h_ms_seq);
    p->h_ms_seq = nullptr;
    if (p->ms_seeded_ev) cudaEventDestroy(p->ms_seeded_ev);
    if (p->join_stream) cudaStreamDestroy(p->join_stream);
    p->d_ms_visited = nullptr;
    p->d_ms_fmask[0] = p->d_ms_fmask[1] = nullptr;
    p->d_ms_labels = nullptr;
    p->d_ms_src = nullptr;
    p->d_ms_depth = nullptr;
    p->d_ms_off = nullptr;
    p->d_ms_join = p->h_ms_join = nullptr;
    p->ms_seeded_ev = nullptr;
    p->join_stream = nullptr;
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
        if ((rc = alloc_dev((void **)&p->d_ms_off, sizeof(int32_t) * 64, "batch level offsets"))) return rc;
        if ((rc = alloc_dev((void **)&p->d_ms_join, sizeof(MsJoin), "batch join requests"))) return rc;
        CUDA_TRY(cudaMallocHost((void **)&p->h_ms_join, sizeof(MsJoin)), "pinned join requests");
        memset(p->h_ms_join, 0, sizeof(MsJoin));
        CUDA_TRY(cudaMallocHost((void **)&p->h_ms_seq, sizeof(int32_t) * 65), "pinned join counts");
        for (int i = 0; i <= 64; i++) p->h_ms_seq[i] = i;
        CUDA_TRY(cudaStreamCreateWithFlags(&p->join_stream, cudaStreamNonBlocking), "join stream");
        CUDA_TRY(cudaEventCreateWithFlags(&p->ms_seeded_ev, cudaEventDisableTiming), "event");
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
    m.level_off = p->d_ms_off;
    m.join = p->d_ms_join;
    m.k = k;
    m.rows = p->ms_labels_k;
    m.pull_ok = p->symmetric == 1 ? 1 : 0;
    const int block = pol.threads;
    const void *kern = block == 128   ? (const void *)dev::msbfs_kernel<128>
                       : block == 512 ? (const void *)dev::msbfs_kernel<512>
                                      : (const void *)dev::msbfs_kernel<256>;
    const size_t smem = block == 128   ? sizeof(dev::MsSmem<128>)
                        : block == 512 ? sizeof(dev::MsSmem<512>)
                                       : sizeof(dev::MsSmem<256>);
    int grid = 0;
    if ((rc = persistent_grid(p, kern, pol, max_grid, smem, &grid))) return rc;
    CUDA_TRY(cudaEventRecord(p->ev0, p->stream), "event record");
    if ((rc = begin_instrumented(p))) return rc;
    // join requests still being copied for an earlier batch land before this
    // batch's seed kernel resets the request block, and their pinned staging
    // entries are read before this batch's requests rewrite them
    if (p->ms_joins > 0) CUDA_TRY(cudaStreamSynchronize(p->join_stream), "join copies");
    const int init_blocks = std::max(1, std::min<int>(p->sms * 8, (int)(((long long)p->nodes + 255) / 256)));
    dev::msbfs_init_kernel<<<init_blocks, kThreads, 0, p->stream>>>(bp, m);
    CUDA_TRY(cudaGetLastError(), "batch init launch");
    dev::msbfs_seed_kernel<<<1, 32, 0, p->stream>>>(bp, m, seed);
    CUDA_TRY(cudaGetLastError(), "batch seed launch");
    // requests for this batch are copied only after its seed kernel
    CUDA_TRY(cudaEventRecord(p->ms_seeded_ev, p->stream), "event record");
    p->ms_joins = 0;
    if ((rc = mark_search_start(p))) return rc;
    void *args[] = {&bp, &m};
    CUDA_TRY(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(block), args, smem, p->stream),
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

int b40c_msbfs_join(b40c_bfs_problem *p, int32_t slot, int32_t source, int32_t depth_limit)
{
    b40c::clear_error();
    if (!p) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null problem");
    if (p->ms_k < 1 || !p->d_ms_join) return b40c::fail(B40C_ERROR_NOT_READY, "no batch has been enacted");
    if (source < 0 || source >= p->nodes) return b40c::fail(B40C_ERROR_INVALID_VALUE, "source %d out of range", source);
    if (slot < p->ms_k || slot >= std::min(64, (int)p->ms_labels_k))
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "join slot %d: must be in [%d, %d) (the batch's k .. label rows)",
                          slot, p->ms_k, std::min(64, (int)p->ms_labels_k));
    if (p->ms_joins >= 64) return b40c::fail(B40C_ERROR_INVALID_VALUE, "at most 64 join requests per batch");
    DeviceGuard guard(p->device);
    // request j's pinned staging entries are written once per batch (the next
    // batch waits for these copies before rewriting them) and the count comes
    // from a constant table, so no copy reads a value changed after it was issued
    MsJoin *h = p->h_ms_join;
    const int j = p->ms_joins;
    h->src[j] = source;
    h->slot[j] = slot;
    h->limit[j] = depth_limit < 0 ? -1 : depth_limit;
    CUDA_TRY(cudaStreamWaitEvent(p->join_stream, p->ms_seeded_ev, 0), "stream wait");
    // the request first, then the count that makes it visible (stream order)
    CUDA_TRY(cudaMemcpyAsync(&p->d_ms_join->src[j], &h->src[j], sizeof(int32_t), cudaMemcpyHostToDevice,
                             p->join_stream),
             "join request copy");
    CUDA_TRY(cudaMemcpyAsync(&p->d_ms_join->slot[j], &h->slot[j], sizeof(int32_t), cudaMemcpyHostToDevice,
                             p->join_stream),
             "join request copy");
    CUDA_TRY(cudaMemcpyAsync(&p->d_ms_join->limit[j], &h->limit[j], sizeof(int32_t), cudaMemcpyHostToDevice,
                             p->join_stream),
             "join request copy");
    CUDA_TRY(cudaMemcpyAsync(&p->d_ms_join->count, p->h_ms_seq + j + 1, sizeof(int32_t), cudaMemcpyHostToDevice,
                             p->join_stream),
             "join count copy");
    p->ms_joins = j + 1;
    return B40C_SUCCESS;
}

int b40c_msbfs_joined(b40c_bfs_problem *p, int32_t *taken, int32_t *search_depths)
{
    b40c::clear_error();
    if (!p || !taken) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    if (p->ms_k < 1 || !p->d_ms_join) return b40c::fail(B40C_ERROR_NOT_READY, "no batch has run");
    DeviceGuard guard(p->device);
    int rc = read_state(p);
    if (rc) return rc;
    if ((rc = check_state_errors(p))) return rc;
    CUDA_TRY(cudaMemcpyAsync(taken, &p->d_ms_join->taken, sizeof(int32_t), cudaMemcpyDeviceToHost, p->stream),
             "join count read");
    if (search_depths)
        CUDA_TRY(cudaMemcpyAsync(search_depths, p->d_ms_depth, sizeof(int32_t) * 64, cudaMemcpyDeviceToHost, p->stream),
                 "batch depth copy");
    CUDA_TRY(cudaStreamSynchronize(p->stream), "join read synchronize");
    return B40C_SUCCESS;
}

int b40c_msbfs_extract(b40c_bfs_problem *p, int slot, int32_t *h_labels)
{
    b40c::clear_error();
    if (!p || !h_labels) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    // slots past k hold the sources sent to join the batch (b40c_msbfs_join)
    if (slot < 0 || slot >= std::min(p->ms_k + p->ms_joins, std::max(p->ms_k, std::min(64, (int)p->ms_labels_k))))
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "no source %d in the last batch", slot);
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
