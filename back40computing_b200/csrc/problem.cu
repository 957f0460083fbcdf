// Problem allocation, policies and the C ABI of the BFS library.
#include <functional>
#include <vector>

#include "bfs_kernels.cuh"
#include "problem.h"

#define B40C_VERSION_STRING "b40c-b200 0.1 (sm_100a)"

using namespace b40c;
using namespace b40c::rt;

namespace b40c {
namespace rt {

int alloc_dev(void **p, size_t bytes, const char *what)
{
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "cudaMalloc %s (%zu bytes) failed: %s", what, bytes,
                          cudaGetErrorString(e));
    }
    return B40C_SUCCESS;
}

void free_vf(VertexFrontier &f)
{
    if (f.v) cudaFree(f.v);
    if (f.col) cudaFree(f.col);
    if (f.P) cudaFree(f.P);
    if (f.cf) cudaFree(f.cf);
    f = VertexFrontier{};
}
void free_ef(EdgeFrontier &f)
{
    if (f.v) cudaFree(f.v);
    if (f.pred) cudaFree(f.pred);
    f = EdgeFrontier{};
}

int ensure_vf(b40c_bfs_problem *p, int i, int64_t cap)
{
    cap = std::max<int64_t>(cap, 1);
    if (p->vcap[i] >= cap) return B40C_SUCCESS;
    free_vf(p->vf[i]);
    p->vcap[i] = 0;
    int rc;
    if ((rc = alloc_dev((void **)&p->vf[i].v, sizeof(int32_t) * cap, "vertex frontier"))) return rc;
    if ((rc = alloc_dev((void **)&p->vf[i].col, sizeof(int32_t) * cap, "vertex frontier"))) return rc;
    if ((rc = alloc_dev((void **)&p->vf[i].P, sizeof(int32_t) * (cap + 1), "vertex frontier"))) return rc;
    // a level's edge total never exceeds m (each vertex is expanded at most once)
    const int64_t cf_len = (std::max<int64_t>(p->edges, 1) + dev::kChunkGrain - 1) / dev::kChunkGrain + 2;
    if ((rc = alloc_dev((void **)&p->vf[i].cf, sizeof(int32_t) * cf_len, "vertex frontier"))) return rc;
    p->vcap[i] = cap;
    return B40C_SUCCESS;
}

int ensure_ef(b40c_bfs_problem *p, int i, int64_t cap)
{
    cap = std::max<int64_t>(cap, 1);
    if (p->ecap[i] >= cap && (!p->mark_pred || p->ef[i].pred)) return B40C_SUCCESS;
    free_ef(p->ef[i]);
    p->ecap[i] = 0;
    int rc;
    if ((rc = alloc_dev((void **)&p->ef[i].v, sizeof(int32_t) * cap, "edge frontier"))) return rc;
    if (p->mark_pred && (rc = alloc_dev((void **)&p->ef[i].pred, sizeof(int32_t) * cap, "edge frontier"))) return rc;
    p->ecap[i] = cap;
    return B40C_SUCCESS;
}

int64_t cap_of(double qs, int64_t base)
{
    double c = std::ceil(qs * (double)base);
    if (c > (double)INT32_MAX - 1) c = (double)INT32_MAX - 1;
    return (int64_t)c;
}

// Look-back slots: one per chunk of the largest possible level.
int ensure_slots(b40c_bfs_problem *p)
{
    const int64_t need = (std::max(p->edges, p->nodes) + 255) / 256 + 4096;
    if (p->max_slots >= need) return B40C_SUCCESS;
    if (p->slots) cudaFree(p->slots);
    p->slots = nullptr;
    p->max_slots = 0;
    int rc = alloc_dev((void **)&p->slots, sizeof(dev::LookbackSlot) * need, "look-back slots");
    if (rc) return rc;
    CUDA_TRY(cudaMemsetAsync(p->slots, 0, sizeof(dev::LookbackSlot) * need, p->stream), "memset look-back slots");
    p->max_slots = (int32_t)need;
    return B40C_SUCCESS;
}

// Test-only: B40C_TEST_SPIN_LIMIT=<polls> shortens every device-side wait of
// the searches enacted from then on, so a test can make one run out quickly.
uint32_t test_spin_limit()
{
    const char *s = getenv("B40C_TEST_SPIN_LIMIT");
    if (!s) return dev::kSpinLimit;
    const long v = atol(s);
    return v > 0 && v < (long)dev::kSpinLimit ? (uint32_t)v : dev::kSpinLimit;
}

BfsParams make_params(b40c_bfs_problem *p, const b40c_bfs_policy &pol)
{
    BfsParams k{};
    k.row_offsets = p->d_ro;
    k.column_indices = p->d_ci;
    k.labels = p->d_labels;
    k.mask = p->d_mask;
    k.iso = p->d_iso;
    k.hub2 = pol.bottom_up_hub_probes > 0 ? (const int2 *)p->d_hub2 : nullptr;
    k.nodes = (int32_t)p->nodes;
    k.edges = (int32_t)p->edges;
    k.mask_words = p->mask_words;
    k.vcap = (int32_t)std::min(p->vcap[0] ? p->vcap[0] : INT32_MAX, p->vcap[1] ? p->vcap[1] : INT32_MAX);
    k.ecap = (int32_t)std::min(p->ecap[0] ? p->ecap[0] : INT32_MAX, p->ecap[1] ? p->ecap[1] : INT32_MAX);
    k.max_chunks = p->max_slots;
    k.cf_cap = (int32_t)((std::max<int64_t>(p->edges, 1) + dev::kChunkGrain - 1) / dev::kChunkGrain + 2);
    k.vf[0] = p->vf[0];
    k.vf[1] = p->vf[1];
    k.ef[0] = p->ef[0];
    k.ef[1] = p->ef[1];
    k.slots = p->slots;
    k.st = p->st;
    k.max_levels = 1;
    k.chunk_edges = pol.chunk_edges;
    k.warp_thresh = pol.warp_gather_threshold;
    k.cta_thresh = pol.cta_gather_threshold;
    k.warp_cull = pol.warp_cull;
    k.precheck = pol.bitmask_precheck > 0 ? pol.bitmask_precheck : 0;  // -1 (off) must not read as true
    k.saturation = pol.saturation_quit;
    k.persistent = 0;
    k.skip_arrival_cta = -1;
    k.spin_limit = test_spin_limit();
    // a host-mapped CSR (stream_from_host) is read with plain loads only
    k.bulk_ok = p->stream_from_host ? 0 : 1;
    k.alloc_lookback = pol.queue_allocation == 1 ? 1 : 0;
    k.direction_opt = 0;
    k.bu_alpha = pol.bottom_up_alpha;
    k.bu_beta = pol.bottom_up_beta;
    k.mask_alt = p->d_next;
    k.small_edges = pol.small_frontier_edges;
    k.subgrid_edges = pol.subgrid_frontier_edges > 0 ? pol.subgrid_frontier_edges : 0;
    k.bu_scan = pol.bottom_up_scan;
    k.bu_long = pol.bottom_up_long_list;
    k.hist_log = pol.history_cull > 0 ? kHistLog : 0;
    // the staged copies need 16-byte aligned device arrays (not a host-mapped CSR)
    k.bu_prefetch = pol.bottom_up_prefetch > 0 && k.bulk_ok && (reinterpret_cast<uintptr_t>(p->d_ro) & 15) == 0 ? 1 : 0;
    k.bu_defer = pol.bottom_up_defer_frontier > 0 ? 1 : 0;
    k.warp_contract = pol.warp_contract > 0 ? 1 : 0;
    k.warp_bu = pol.warp_bottom_up > 0 ? 1 : 0;
    k.levels = p->instrument ? p->d_levels : nullptr;
    k.duty = p->instrument ? p->d_duty : nullptr;
    k.arrive = p->instrument ? p->d_arrive : nullptr;
    k.cond_handle = 0;
    return k;
}

b40c_bfs_policy default_policy(int strategy)
{
    b40c_bfs_policy pol{};
    pol.threads = kThreads;
    pol.ctas_per_sm = 0;
    pol.chunk_edges = dev::kChunkMax;
    pol.warp_gather_threshold = 32;
    pol.cta_gather_threshold = 512;
    pol.saturation_quit = 512;  // SATURATION_QUIT = 4 * 128 (enactor_hybrid.cuh:571)
    pol.warp_cull = 0;
    pol.bitmask_precheck = 1;
    pol.bottom_up_alpha = 14;  // Beamer et al.'s defaults
    pol.bottom_up_beta = 24;
    pol.small_frontier_edges = 1024;
    pol.bottom_up_scan = 1;
    pol.bottom_up_hub_probes = 1;
    pol.bottom_up_list = -1;
    pol.bottom_up_defer_frontier = 1;
    pol.subgrid_frontier_edges = -1;
    pol.bottom_up_long_list = 256;
    pol.history_cull = -1;
    pol.queue_allocation = 2;  // measured faster than look-back on RMAT-22 (1.75 vs 2.29 ms)
    pol.warp_contract = 1;
    pol.warp_bottom_up = 1;
    if (strategy == B40C_DIRECTION_OPTIMIZING) {
        // measured on B200 over 16 sources: the kernel variant carrying the
        // unvisited lists is slower overall (R-MAT 22 241 vs 222 us, random
        // 2^21 203 vs 172 us: its first bottom-up level loses more than the
        // later ones gain), so lists stay off; the visited-word pre-check
        // makes no difference here
        pol.bottom_up_list = -1;
        pol.bitmask_precheck = -1;
    }
    return pol;
}

int resolve_policy(int strategy, const b40c_bfs_policy *in, b40c_bfs_policy *out)
{
    b40c_bfs_policy d = default_policy(strategy);
    if (in) {
        if (in->threads) d.threads = in->threads;
        if (in->ctas_per_sm) d.ctas_per_sm = in->ctas_per_sm;
        if (in->chunk_edges) d.chunk_edges = in->chunk_edges;
        if (in->warp_gather_threshold) d.warp_gather_threshold = in->warp_gather_threshold;
        if (in->cta_gather_threshold) d.cta_gather_threshold = in->cta_gather_threshold;
        if (in->saturation_quit) d.saturation_quit = in->saturation_quit;
        if (in->warp_cull) d.warp_cull = in->warp_cull > 0 ? 1 : 0;
        if (in->bitmask_precheck) d.bitmask_precheck = in->bitmask_precheck > 0 ? std::min(in->bitmask_precheck, 2) : -1;
        if (in->queue_allocation) d.queue_allocation = in->queue_allocation;
        if (in->bottom_up_alpha) d.bottom_up_alpha = in->bottom_up_alpha;
        if (in->bottom_up_beta) d.bottom_up_beta = in->bottom_up_beta;
        if (in->small_frontier_edges) d.small_frontier_edges = in->small_frontier_edges;
        if (in->bottom_up_scan) d.bottom_up_scan = in->bottom_up_scan;
        if (in->bottom_up_hub_probes) d.bottom_up_hub_probes = in->bottom_up_hub_probes > 0 ? 1 : -1;
        if (in->bottom_up_list) d.bottom_up_list = in->bottom_up_list > 0 ? 1 : -1;
        if (in->bottom_up_defer_frontier) d.bottom_up_defer_frontier = in->bottom_up_defer_frontier > 0 ? 1 : -1;
        if (in->subgrid_frontier_edges) d.subgrid_frontier_edges = in->subgrid_frontier_edges > 0 ? in->subgrid_frontier_edges : -1;
        if (in->bottom_up_long_list) d.bottom_up_long_list = in->bottom_up_long_list;
        if (in->history_cull) d.history_cull = in->history_cull > 0 ? 1 : -1;
        if (in->bottom_up_prefetch) d.bottom_up_prefetch = in->bottom_up_prefetch > 0 ? 1 : -1;
        if (in->warp_contract) d.warp_contract = in->warp_contract > 0 ? 1 : -1;
        if (in->warp_bottom_up) d.warp_bottom_up = in->warp_bottom_up > 0 ? 1 : -1;
    }
    if (d.threads != 128 && d.threads != 256 && d.threads != 512)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.threads %d not built (available: 128, 256, 512)",
                          d.threads);
    if (d.chunk_edges < 256 || d.chunk_edges > dev::kChunkMax || (d.chunk_edges & 31))
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.chunk_edges must be a multiple of 32 in [256, %d]",
                          dev::kChunkMax);
    if (d.warp_gather_threshold < 32)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.warp_gather_threshold must be >= 32");
    if (d.cta_gather_threshold < 32)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.cta_gather_threshold must be >= 32");
    if (d.queue_allocation != 1 && d.queue_allocation != 2)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.queue_allocation must be 1 (look-back) or 2 (atomic)");
    if (d.bottom_up_alpha < 1 || d.bottom_up_beta < 1)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.bottom_up_alpha and bottom_up_beta must be >= 1");
    if (d.saturation_quit < 1) return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.saturation_quit must be >= 1");
    if (d.bottom_up_scan != 1)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.bottom_up_scan must be 1 (per-lane list scans)");
    if (d.ctas_per_sm < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.ctas_per_sm must be >= 0");
    // the prefetch buffer serves the CTA-wide first bottom-up level only (the
    // warp-autonomous one reads straight from global memory)
    if (d.bottom_up_prefetch == 0) d.bottom_up_prefetch = d.threads >= 512 && d.warp_bottom_up < 0 ? 1 : -1;
    if (d.bottom_up_long_list < 4)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "policy.bottom_up_long_list must be >= 4");
    *out = d;
    return B40C_SUCCESS;
}

// Device bytes a handle holds right now (the sizes its allocations asked
// for; alloc_dev asks for at least 16 bytes).
int64_t device_bytes(const b40c_bfs_problem *p)
{
    auto a = [](int64_t b) { return std::max<int64_t>(b, 16); };
    const int64_t n = p->nodes, m = p->edges;
    int64_t t = 0;
    if (p->own_csr && p->d_ro) t += a(4 * (n + 1)) + a(4 * std::max<int64_t>(m, 1));
    if (p->d_labels) t += a(4 * n);
    const int64_t mask = a(4 * ((int64_t)(p->mask_words + 63) / 64 * 64));
    if (p->d_mask) t += mask;
    if (p->d_iso) t += mask;
    if (p->d_hub2) t += a(8 * n);
    for (int i = 0; i < 2; i++)
        if (p->d_ul[i]) t += a(4 * n);
    if (p->d_next) t += mask;
    if (p->st) t += a(sizeof(SearchState));
    if (p->slots) t += a((int64_t)sizeof(dev::LookbackSlot) * p->max_slots);
    const int64_t cf_len = (std::max<int64_t>(m, 1) + dev::kChunkGrain - 1) / dev::kChunkGrain + 2;
    for (int i = 0; i < 2; i++) {
        if (p->vcap[i]) t += 2 * a(4 * p->vcap[i]) + a(4 * (p->vcap[i] + 1)) + a(4 * cf_len);
        if (p->ecap[i]) t += a(4 * p->ecap[i]) * (p->ef[i].pred ? 2 : 1);
    }
    if (p->d_ms_visited) t += 3 * a(8 * n) + 2 * a(4 * 64);
    if (p->d_ms_labels) t += a(4 * n * (int64_t)p->ms_labels_k);
    if (p->d_levels) t += a((int64_t)sizeof(LevelRecord) * kMaxLevelRecords);
    if (p->d_duty) t += a(4 * sizeof(unsigned long long));
    if (p->d_arrive) t += a((int64_t)sizeof(unsigned long long) * kMaxArrivePasses * kMaxArriveCtas * kPhaseStamps);
    for (int i = 0; i < 2; i++)
        if (p->d_stage[i]) t += a(4 * n);
    if (p->d_stage_err) t += a(8);
    return t;
}

// What a handle built from a host CSR (copied to the device) holds after a
// batched search of width k and a single-source vertex-frontier search with
// queue sizing qs: device_bytes() of that handle, computed without one.
int64_t planned_bytes(int64_t n, int64_t m, int k, double qs)
{
    auto a = [](int64_t b) { return std::max<int64_t>(b, 16); };
    const int64_t mask_words = (n + 31) / 32;
    const int64_t mask = a(4 * ((mask_words + 63) / 64 * 64));
    const int64_t slots = (std::max(m, n) + 255) / 256 + 4096;
    const int64_t cap = std::max<int64_t>(cap_of(qs, n), 1);
    const int64_t cf_len = (std::max<int64_t>(m, 1) + dev::kChunkGrain - 1) / dev::kChunkGrain + 2;
    int64_t t = a(4 * (n + 1)) + a(4 * std::max<int64_t>(m, 1));
    t += a(4 * n) + 3 * mask + a(sizeof(SearchState)) + a((int64_t)sizeof(dev::LookbackSlot) * slots);
    t += 2 * (2 * a(4 * cap) + a(4 * (cap + 1)) + a(4 * cf_len));
    t += a(8 * n);      // hub pairs (built by the server for every graph)
    t += 2 * a(4 * n);  // unvisited lists (direction-optimizing distance searches)
    if (k > 0) t += 3 * a(8 * n) + 2 * a(4 * 64) + a(4 * n * (int64_t)k);
    return t;
}

// Reads the device state into the pinned mirror (synchronous).
int read_state(b40c_bfs_problem *p)
{
    CUDA_TRY(cudaMemcpyAsync(p->h_st, p->st, sizeof(SearchState), cudaMemcpyDeviceToHost, p->stream), "state read");
    CUDA_TRY(cudaStreamSynchronize(p->stream), "stream synchronize");
    return B40C_SUCCESS;
}

int error_status(unsigned e)
{
    if (e & dev::kErrOverflow)
        return b40c::fail(B40C_ERROR_INVALID_CONFIGURATION,
                          "Frontier queue overflow.  Please increase queue-sizing factor.");
    if (e & dev::kErrLevels)
        return b40c::fail(B40C_ERROR_LAUNCH_TIMEOUT, "a replayed search ran more levels than the graph has vertices");
    if (e & dev::kErrFrontier)
        return b40c::fail(B40C_ERROR_INTERNAL, "a deferred bottom-up frontier did not match its counted size");
    if (e & (dev::kErrBarrier | dev::kErrLookback | dev::kErrBulk))
        return b40c::fail(B40C_ERROR_LAUNCH_TIMEOUT, "a bounded device-side wait expired (error bits 0x%x)", e);
    return B40C_SUCCESS;
}

int check_state_errors(b40c_bfs_problem *p) { return error_status(p->h_st->error); }

// Copies labels[n] into a staging slot (16-byte vectors; cudaMalloc'd buffers
// are aligned) and the search's error word beside it.
__global__ void stage_results_kernel(const int32_t *labels, int32_t *stage, int64_t n, const uint32_t *err,
                                     uint32_t *err_out)
{
    const int64_t n4 = n / 4;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int4 *src4 = reinterpret_cast<const int4 *>(labels);
    int4 *dst4 = reinterpret_cast<int4 *>(stage);
    for (int64_t i = t0; i < n4; i += stride) dst4[i] = src4[i];
    for (int64_t i = 4 * n4 + t0; i < n; i += stride) stage[i] = labels[i];
    if (t0 == 0) *err_out = *err;
}


int persistent_grid(b40c_bfs_problem *p, const void *kernel, const b40c_bfs_policy &pol, int max_grid,
                            size_t smem, int *grid)
{
    int per_sm = 0;
    CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, pol.threads, smem), "occupancy query");
    if (per_sm < 1) return b40c::fail(B40C_ERROR_INVALID_CONFIGURATION, "kernel cannot be resident");
    if (pol.ctas_per_sm > 0) per_sm = std::min(per_sm, pol.ctas_per_sm);
    int g = per_sm * p->sms;
    if (max_grid > 0) g = std::min(g, max_grid);
    *grid = std::max(g, 1);
    p->last_grid = *grid;
    return B40C_SUCCESS;
}

int finish_timing(b40c_bfs_problem *p)
{
    CUDA_TRY(cudaEventRecord(p->ring_b[p->ring_pos], p->stream), "event record");
    CUDA_TRY(cudaEventRecord(p->ev1, p->stream), "event record");
    p->ring_pos = (p->ring_pos + 1) % b40c_bfs_problem::kRing;
    p->ring_count = std::min(p->ring_count + 1, b40c_bfs_problem::kRing);
    p->timed = true;
    return B40C_SUCCESS;
}


// Edgeless vertices (no out-edges and no in-edges, so on a directed graph too
// nothing can reach them): first each word gets the bits of vertices with
// out-edges, then every edge sets its head's bit, then the words are inverted.
__global__ void out_edge_mask_kernel(const int32_t *ro, int32_t nodes, uint32_t *bits, int32_t words)
{
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
        uint32_t b = 0;
        for (int k = 0; k < 32; k++) {
            const int v = w * 32 + k;
            if (v < nodes && ro[v + 1] > ro[v]) b |= 1u << k;
        }
        bits[w] = b;
    }
}

__global__ void in_edge_mask_kernel(const int32_t *ci, int64_t edges, uint32_t *bits)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < edges; e += stride) {
        const int u = ci[e];
        const uint32_t bit = 1u << (u & 31);
        if (!(bits[u >> 5] & bit)) atomicOr(bits + (u >> 5), bit);
    }
}

__global__ void invert_mask_kernel(uint32_t *bits, int32_t nodes, int32_t words)
{
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
        const int left = nodes - w * 32;
        const uint32_t valid = left >= 32 ? 0xffffffffu : ((1u << left) - 1u);
        bits[w] = ~bits[w] & valid;
    }
}

// Order-independent fingerprints of the edge multiset and of its reversal:
// sums of a 64-bit mix (splitmix64's finaliser) of (u << 32 | v) and of
// (v << 32 | u).  Equal sums <=> symmetric, up to a 2^-64 collision chance.
__global__ void symmetry_hash_kernel(const int32_t *ro, const int32_t *ci, int32_t nodes, unsigned long long *sums)
{
    auto mix = [](unsigned long long z) {
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long fwd = 0, rev = 0;
    for (int u = warp; u < nodes; u += nwarps) {
        for (int e = ro[u] + lane; e < ro[u + 1]; e += 32) {
            const unsigned long long v = (unsigned)ci[e];
            fwd += mix(((unsigned long long)(unsigned)u << 32) | v);
            rev += mix((v << 32) | (unsigned)u);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        fwd += __shfl_down_sync(0xffffffffu, fwd, off);
        rev += __shfl_down_sync(0xffffffffu, rev, off);
    }
    if (lane == 0) {
        atomicAdd(&sums[0], fwd);
        atomicAdd(&sums[1], rev);
    }
}

int check_symmetric(b40c_bfs_problem *p)
{
    if (p->symmetric >= 0) return B40C_SUCCESS;
    unsigned long long *d_sums = nullptr;
    int rc = alloc_dev((void **)&d_sums, 2 * sizeof(unsigned long long), "symmetry sums");
    if (rc) return rc;
    unsigned long long h[2] = {1, 2};
    cudaError_t e = cudaMemsetAsync(d_sums, 0, 2 * sizeof(unsigned long long), p->stream);
    if (e == cudaSuccess) {
        symmetry_hash_kernel<<<p->sms * 8, 256, 0, p->stream>>>(p->d_ro, p->d_ci, (int32_t)p->nodes, d_sums);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_sums, sizeof(h), cudaMemcpyDeviceToHost, p->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    cudaFree(d_sums);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return b40c::fail((int)e, "symmetry check failed: %s", cudaGetErrorString(e));
    }
    p->symmetric = h[0] == h[1] ? 1 : 0;
    return B40C_SUCCESS;
}

// Per vertex v, its two highest-degree distinct neighbours other than v
// (ties: the smaller id), -1 where it has fewer.  One warp per vertex; each
// lane keeps its own best two, then two warp arg-max rounds pick the pair.
// Bottom-up levels probe this pair first: on power-law graphs a vertex's hub
// neighbours are the ones most likely to be in the frontier.
__device__ __forceinline__ unsigned long long hub_key(int deg, int id)
{
    return ((unsigned long long)(unsigned)deg << 32) | (unsigned)(0x7fffffff - id);
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long x)
{
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
        x = y > x ? y : x;
    }
    return x;
}

__global__ void hub_pair_kernel(const int32_t *ro, const int32_t *ci, int32_t nodes, int2 *hub)
{
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nodes; v += nwarps) {
        const int r0 = ro[v], r1 = ro[v + 1];
        unsigned long long b1 = 0, b2 = 0;  // 0 = none (a real key has a nonzero id part)
        for (int e = r0 + lane; e < r1; e += 32) {
            const int u = ci[e];
            if (u == v) continue;
            const unsigned long long k = hub_key(ro[u + 1] - ro[u], u);
            if (k == b1 || k == b2) continue;  // duplicate edge
            if (k > b1) {
                b2 = b1;
                b1 = k;
            } else if (k > b2) {
                b2 = k;
            }
        }
        const unsigned long long m1 = warp_max_u64(b1);
        const unsigned long long m2 = warp_max_u64(b1 == m1 ? b2 : b1);
        if (lane == 0) {
            int2 h;
            h.x = m1 ? 0x7fffffff - (int)(unsigned)(m1 & 0xffffffffu) : -1;
            h.y = m2 ? 0x7fffffff - (int)(unsigned)(m2 & 0xffffffffu) : -1;
            hub[v] = h;
        }
    }
}

// Builds the hub pairs of a symmetric problem once (8 bytes per vertex).
int ensure_hubs(b40c_bfs_problem *p)
{
    if (p->d_hub2) return B40C_SUCCESS;
    int rc = alloc_dev((void **)&p->d_hub2, sizeof(int2) * (size_t)p->nodes, "hub pairs");
    if (rc) return rc;
    const int blocks = std::max(1, std::min<int>(p->sms * 16, (int)((p->nodes * 32 + 255) / 256)));
    hub_pair_kernel<<<blocks, 256, 0, p->stream>>>(p->d_ro, p->d_ci, (int32_t)p->nodes, (int2 *)p->d_hub2);
    CUDA_TRY(cudaGetLastError(), "hub pair launch");
    return B40C_SUCCESS;
}

// The two unvisited-vertex lists of bottom-up list mode (4 bytes per vertex each).
int ensure_unvisited_lists(b40c_bfs_problem *p)
{
    for (int i = 0; i < 2; i++)
        if (!p->d_ul[i]) {
            int rc = alloc_dev((void **)&p->d_ul[i], sizeof(int32_t) * (size_t)p->nodes, "unvisited list");
            if (rc) return rc;
        }
    return B40C_SUCCESS;
}

// Clears the instrumentation buffers before an instrumented search.
int begin_instrumented(b40c_bfs_problem *p)
{
    if (!p->instrument) return B40C_SUCCESS;
    CUDA_TRY(cudaMemsetAsync(p->d_levels, 0, sizeof(LevelRecord) * kMaxLevelRecords, p->stream), "level records reset");
    CUDA_TRY(cudaMemsetAsync(p->d_duty, 0, 4 * sizeof(unsigned long long), p->stream), "duty reset");
    CUDA_TRY(cudaMemsetAsync(p->d_arrive, 0, sizeof(unsigned long long) * kMaxArrivePasses * kMaxArriveCtas * kPhaseStamps,
                             p->stream),
             "arrival reset");
    return B40C_SUCCESS;
}

void free_graphs(b40c_bfs_problem *p)
{
    for (int s = 0; s < 5; s++) {
        if (p->graph_exec[s]) cudaGraphExecDestroy(p->graph_exec[s]);
        if (p->graph_def[s]) cudaGraphDestroy(p->graph_def[s]);
        p->graph_exec[s] = nullptr;
        p->graph_def[s] = nullptr;
        p->graph_copy_node[s] = nullptr;
    }
}

int run_graph(b40c_bfs_problem *p, int slot, const KernelNode &init, KernelNode *body, int n_body)
{
    if (!p->graph_exec[slot] || memcmp(&p->graph_params[slot], &body[0].params, sizeof(BfsParams)) != 0 ||
        p->graph_grid[slot] != (int)body[0].grid.x) {
        if (p->graph_exec[slot]) cudaGraphExecDestroy(p->graph_exec[slot]);
        if (p->graph_def[slot]) cudaGraphDestroy(p->graph_def[slot]);
        p->graph_exec[slot] = nullptr;
        p->graph_def[slot] = nullptr;
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaGraphCreate(&g, 0), "cudaGraphCreate");
        p->graph_def[slot] = g;  // owned by the handle from here on (free_graphs)
        cudaGraphNode_t n_copy, n_init, n_loop;
        CUDA_TRY(cudaGraphAddMemcpyNode1D(&n_copy, g, nullptr, 0, &p->st->src, source_slot(p), 2 * sizeof(int32_t),
                                          cudaMemcpyHostToDevice),
                 "graph memcpy node");
        p->graph_copy_node[slot] = n_copy;
        BfsParams init_params = init.params;
        void *init_args[] = {&init_params};
        cudaKernelNodeParams kp = {};
        kp.func = (void *)init.func;
        kp.gridDim = init.grid;
        kp.blockDim = init.block;
        kp.sharedMemBytes = (unsigned)init.smem;
        kp.kernelParams = init_args;
        CUDA_TRY(cudaGraphAddKernelNode(&n_init, g, &n_copy, 1, &kp), "graph init node");
        cudaGraphConditionalHandle handle;
        CUDA_TRY(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault),
                 "cudaGraphConditionalHandleCreate");
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        CUDA_TRY(cudaGraphAddNode(&n_loop, g, &n_init, 1, &cp), "graph WHILE node");
        cudaGraph_t loop_body = cp.conditional.phGraph_out[0];
        cudaGraphNode_t prev = nullptr;
        for (int i = 0; i < n_body; i++) {
            BfsParams bp = body[i].params;
            bp.cond_handle = (i == n_body - 1) ? (unsigned long long)handle : 0ull;
            void *args[] = {&bp};
            cudaKernelNodeParams kb = {};
            kb.func = (void *)body[i].func;
            kb.gridDim = body[i].grid;
            kb.blockDim = body[i].block;
            kb.sharedMemBytes = (unsigned)body[i].smem;
            kb.kernelParams = args;
            cudaGraphNode_t n;
            CUDA_TRY(cudaGraphAddKernelNode(&n, loop_body, prev ? &prev : nullptr, prev ? 1 : 0, &kb), "graph body node");
            prev = n;
        }
        CUDA_TRY(cudaGraphInstantiate(&p->graph_exec[slot], g, 0), "cudaGraphInstantiate");
        p->graph_params[slot] = body[0].params;
        p->graph_grid[slot] = (int)body[0].grid.x;
    } else {
        // this launch's source pair lives in its own ring slot
        CUDA_TRY(cudaGraphExecMemcpyNodeSetParams1D(p->graph_exec[slot], p->graph_copy_node[slot], &p->st->src,
                                                    source_slot(p), 2 * sizeof(int32_t), cudaMemcpyHostToDevice),
                 "graph source re-point");
    }
    CUDA_TRY(cudaGraphLaunch(p->graph_exec[slot], p->stream), "cudaGraphLaunch");
    return B40C_SUCCESS;
}

}  // namespace rt
}  // namespace b40c

namespace b40c {
namespace rt {

int create_problem(int64_t nodes, int64_t edges, int mark_pred, int stream_from_host, int device,
                   const std::function<int(b40c_bfs_problem *)> &load, b40c_bfs_problem **out)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return b40c::fail(B40C_ERROR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return b40c::fail(B40C_ERROR_NO_DEVICE, "no current CUDA device");
    }
    if (device >= ndev) return b40c::fail(B40C_ERROR_INVALID_VALUE, "invalid device %d", device);
    DeviceGuard guard(device);
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (prop.major != 10)
        return b40c::fail(B40C_ERROR_INVALID_DEVICE_FUNCTION, "kernels are built for sm_100a; device is sm_%d%d",
                          prop.major, prop.minor);
    auto *p = new b40c_bfs_problem();
    p->device = device;
    p->nodes = nodes;
    p->edges = edges;
    p->mark_pred = mark_pred ? 1 : 0;
    p->stream_from_host = stream_from_host ? 1 : 0;
    p->sms = prop.multiProcessorCount;
    int rc = B40C_SUCCESS;
    auto bail = [&](int code) {
        b40c_bfs_problem_destroy(p);
        return code;
    };
    if (cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return bail(b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "stream creation failed"));
    }
    p->stream = p->own_stream;
    if (cudaEventCreate(&p->ev0) != cudaSuccess || cudaEventCreate(&p->ev1) != cudaSuccess) {
        cudaGetLastError();
        return bail(b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "event creation failed"));
    }
    for (int i = 0; i < b40c_bfs_problem::kRing; i++)
        if (cudaEventCreate(&p->ring_a[i]) != cudaSuccess || cudaEventCreate(&p->ring_b[i]) != cudaSuccess) {
            cudaGetLastError();
            return bail(b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "event creation failed"));
        }
    if ((rc = load(p))) return bail(rc);
    p->mask_words = (int32_t)((nodes + 31) / 32);
    if ((rc = alloc_dev((void **)&p->d_labels, sizeof(int32_t) * nodes, "labels"))) return bail(rc);
    if ((rc = alloc_dev((void **)&p->d_mask, sizeof(uint32_t) * ((p->mask_words + 63) / 64 * 64), "visited mask")))
        return bail(rc);
    // second mask buffer: written whole by a bottom-up level before anything reads it
    if ((rc = alloc_dev((void **)&p->d_next, sizeof(uint32_t) * ((p->mask_words + 63) / 64 * 64), "second mask")))
        return bail(rc);
    // vertices without edges: never reached, never anyone's neighbour; marking
    // them visited up front lets bottom-up levels skip them by the word test
    if ((rc = alloc_dev((void **)&p->d_iso, sizeof(uint32_t) * ((p->mask_words + 63) / 64 * 64), "edgeless mask")))
        return bail(rc);
    {
        const int wb = std::max(1, std::min<int>(p->sms * 8, (p->mask_words + 255) / 256));
        out_edge_mask_kernel<<<wb, 256, 0, p->stream>>>(p->d_ro, (int32_t)nodes, p->d_iso, p->mask_words);
        if (edges > 0)
            in_edge_mask_kernel<<<p->sms * 8, 256, 0, p->stream>>>(p->d_ci, edges, p->d_iso);
        invert_mask_kernel<<<wb, 256, 0, p->stream>>>(p->d_iso, (int32_t)nodes, p->mask_words);
        if (cudaGetLastError() != cudaSuccess)
            return bail(b40c::fail(B40C_ERROR_INVALID_CONFIGURATION, "edgeless mask launch"));
    }
    if ((rc = alloc_dev((void **)&p->st, sizeof(SearchState), "search state"))) return bail(rc);
    if (cudaMemsetAsync(p->st, 0, sizeof(SearchState), p->stream) != cudaSuccess ||
        cudaMallocHost((void **)&p->h_st, sizeof(SearchState)) != cudaSuccess) {
        cudaGetLastError();
        return bail(b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "state allocation failed"));
    }
    memset(p->h_st, 0, sizeof(SearchState));
    if (cudaMallocHost((void **)&p->h_src_ring, 2 * sizeof(int32_t) * b40c_bfs_problem::kRing) != cudaSuccess) {
        cudaGetLastError();
        p->h_src_ring = nullptr;
        return bail(b40c::fail(B40C_ERROR_MEMORY_ALLOCATION, "pinned source ring allocation failed"));
    }
    if ((rc = ensure_slots(p))) return bail(rc);
    if (cudaStreamSynchronize(p->stream) != cudaSuccess) {
        cudaError_t e = cudaGetLastError();
        return bail(b40c::fail((int)e, "problem setup failed: %s", cudaGetErrorString(e)));
    }
    *out = p;
    return B40C_SUCCESS;
}

}  // namespace rt
}  // namespace b40c


// ---- C ABI -----------------------------------------------------------------------------

extern "C" {

const char *b40c_last_error_string(void) { return b40c::error_buffer(); }

const char *b40c_version(void) { return B40C_VERSION_STRING; }

int b40c_device_count(int *count)
{
    b40c::clear_error();
    if (!count) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null count");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c = 0;
    }
    *count = c;
    return B40C_SUCCESS;
}

int b40c_bfs_default_policy(int strategy, b40c_bfs_policy *policy)
{
    b40c::clear_error();
    if (!policy) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null policy");
    if (strategy < B40C_EXPAND_CONTRACT || strategy > B40C_DIRECTION_OPTIMIZING)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "unknown strategy %d", strategy);
    *policy = default_policy(strategy);
    return B40C_SUCCESS;
}

int b40c_bfs_problem_create(const int32_t *h_ro, const int32_t *h_ci, int64_t nodes, int64_t edges, int mark_pred,
                            int stream_from_host, int device, b40c_bfs_problem **out)
{
    b40c::clear_error();
    if (!out) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null output handle");
    *out = nullptr;
    if (!h_ro || (!h_ci && edges > 0) || nodes <= 0 || edges < 0 || nodes >= (int64_t)1 << 30 ||
        edges >= (int64_t)INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE,
                          "invalid CSR (nodes %lld, edges %lld; need 0 < nodes < 2^30, edges < 2^31)", (long long)nodes,
                          (long long)edges);
    // int32 arrays at an address that is not 4-byte aligned cannot be read by
    // the kernels when mapped zero-copy (and are not int32 arrays in C anyway)
    if ((reinterpret_cast<uintptr_t>(h_ro) | reinterpret_cast<uintptr_t>(h_ci)) & 3u)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "row_offsets and column_indices must be 4-byte aligned");
    if (h_ro[0] != 0 || h_ro[nodes] != edges)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "row_offsets must start at 0 and end at edges");
    // the kernels index labels and the mask by column value: reject malformed CSR up front
    for (int64_t v = 0; v < nodes; v++)
        if (h_ro[v + 1] < h_ro[v])
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "row_offsets decrease at vertex %lld", (long long)v);
    for (int64_t e = 0; e < edges; e++)
        if ((uint32_t)h_ci[e] >= (uint32_t)nodes)
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "column index %d at edge %lld out of range", h_ci[e],
                              (long long)e);
    auto load = [&](b40c_bfs_problem *p) -> int {
        if (p->stream_from_host) {
            // zero-copy: the kernels read the caller's host arrays over the bus
            // (csr_problem.cuh:351-363); pin them in place when they are not pinned yet
            const void *arrs[2] = {h_ro, h_ci};
            const size_t bytes[2] = {sizeof(int32_t) * (size_t)(nodes + 1),
                                     sizeof(int32_t) * (size_t)std::max<int64_t>(edges, 1)};
            int32_t **dst[2] = {&p->d_ro, &p->d_ci};
            for (int i = 0; i < 2; i++) {
                cudaPointerAttributes attr;
                cudaError_t e = cudaPointerGetAttributes(&attr, arrs[i]);
                if (e != cudaSuccess || attr.type != cudaMemoryTypeHost) {
                    cudaGetLastError();
                    e = cudaHostRegister((void *)arrs[i], bytes[i], cudaHostRegisterMapped | cudaHostRegisterReadOnly);
                    if (e != cudaSuccess) {
                        cudaGetLastError();
                        return b40c::fail((int)e, "cudaHostRegister for stream-from-host failed: %s",
                                          cudaGetErrorString(e));
                    }
                    (i == 0 ? p->reg_ro : p->reg_ci) = arrs[i];
                }
                e = cudaHostGetDevicePointer((void **)dst[i], (void *)arrs[i], 0);
                if (e != cudaSuccess) {
                    cudaGetLastError();
                    return b40c::fail((int)e, "cudaHostGetDevicePointer failed: %s", cudaGetErrorString(e));
                }
            }
            p->own_csr = false;
            return B40C_SUCCESS;
        }
        int rc;
        if ((rc = alloc_dev((void **)&p->d_ro, sizeof(int32_t) * (nodes + 1), "row offsets"))) return rc;
        if ((rc = alloc_dev((void **)&p->d_ci, sizeof(int32_t) * std::max<int64_t>(edges, 1), "column indices")))
            return rc;
        if (cudaMemcpyAsync(p->d_ro, h_ro, sizeof(int32_t) * (nodes + 1), cudaMemcpyHostToDevice, p->stream) !=
                cudaSuccess ||
            (edges > 0 &&
             cudaMemcpyAsync(p->d_ci, h_ci, sizeof(int32_t) * edges, cudaMemcpyHostToDevice, p->stream) != cudaSuccess)) {
            cudaGetLastError();
            return b40c::fail(B40C_ERROR_INVALID_VALUE, "CSR upload failed");
        }
        return B40C_SUCCESS;
    };
    return rt::create_problem(nodes, edges, mark_pred, stream_from_host, device, load, out);
}

int b40c_bfs_problem_destroy(b40c_bfs_problem *p)
{
    b40c::clear_error();
    if (!p) return B40C_SUCCESS;
    DeviceGuard guard(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    free_graphs(p);
    if (p->own_csr) {
        if (p->d_ro) cudaFree(p->d_ro);
        if (p->d_ci) cudaFree(p->d_ci);
    }
    if (p->reg_ro) cudaHostUnregister((void *)p->reg_ro);
    if (p->reg_ci) cudaHostUnregister((void *)p->reg_ci);
    if (p->d_labels) cudaFree(p->d_labels);
    if (p->d_mask) cudaFree(p->d_mask);
    if (p->d_iso) cudaFree(p->d_iso);
    if (p->d_hub2) cudaFree(p->d_hub2);
    for (int i = 0; i < 2; i++)
        if (p->d_ul[i]) cudaFree(p->d_ul[i]);
    if (p->d_next) cudaFree(p->d_next);
    free_batch(p);
    if (p->d_levels) cudaFree(p->d_levels);
    if (p->d_duty) cudaFree(p->d_duty);
    if (p->d_arrive) cudaFree(p->d_arrive);
    if (p->copy_stream) cudaStreamSynchronize(p->copy_stream);
    for (int i = 0; i < 2; i++) {
        if (p->d_stage[i]) cudaFree(p->d_stage[i]);
        if (p->staged_ev[i]) cudaEventDestroy(p->staged_ev[i]);
        if (p->landed_ev[i]) cudaEventDestroy(p->landed_ev[i]);
    }
    if (p->d_stage_err) cudaFree(p->d_stage_err);
    if (p->h_stage_err) cudaFreeHost(p->h_stage_err);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    for (int i = 0; i < 2; i++) {
        free_vf(p->vf[i]);
        free_ef(p->ef[i]);
    }
    if (p->slots) cudaFree(p->slots);
    if (p->st) cudaFree(p->st);
    if (p->h_st) cudaFreeHost(p->h_st);
    if (p->h_src_ring) cudaFreeHost(p->h_src_ring);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    for (int i = 0; i < b40c_bfs_problem::kRing; i++) {
        if (p->ring_a[i]) cudaEventDestroy(p->ring_a[i]);
        if (p->ring_b[i]) cudaEventDestroy(p->ring_b[i]);
    }
    if (p->own_stream) cudaStreamDestroy(p->own_stream);
    cudaGetLastError();
    delete p;
    return B40C_SUCCESS;
}

int b40c_bfs_problem_device_bytes(b40c_bfs_problem *p, int64_t *bytes)
{
    b40c::clear_error();
    if (!p || !bytes) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    *bytes = device_bytes(p);
    return B40C_SUCCESS;
}

int b40c_bfs_set_stream(b40c_bfs_problem *p, void *stream)
{
    b40c::clear_error();
    if (!p) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null problem");
    p->stream = stream ? (cudaStream_t)stream : p->own_stream;
    return B40C_SUCCESS;
}

int b40c_bfs_problem_reset(b40c_bfs_problem *p, int frontier_type, double queue_sizing)
{
    b40c::clear_error();
    if (!p) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null problem");
    if (frontier_type < B40C_VERTEX_FRONTIERS || frontier_type > B40C_MULTI_GPU_FRONTIERS)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "unknown frontier type %d", frontier_type);
    if (!(queue_sizing > 0.0)) queue_sizing = 1.3;  // "0.0 is unspecified" (csr_problem.cuh:549)
    DeviceGuard guard(p->device);
    p->queue_sizing = queue_sizing;
    int rc;
    const int64_t vc = cap_of(queue_sizing, p->nodes), ec = cap_of(queue_sizing, p->edges);
    switch (frontier_type) {
    case B40C_VERTEX_FRONTIERS:
        if ((rc = ensure_vf(p, 0, vc)) || (rc = ensure_vf(p, 1, vc))) return rc;
        break;
    case B40C_EDGE_FRONTIERS:
        if ((rc = ensure_ef(p, 0, ec)) || (rc = ensure_ef(p, 1, ec))) return rc;
        break;
    default:  // MIXED (and MULTI_GPU, single GPU here)
        if ((rc = ensure_vf(p, 0, vc)) || (rc = ensure_ef(p, 0, ec))) return rc;
        break;
    }
    // labels <- -1, visited mask <- 0 (csr_problem.cuh:723-745)
    CUDA_TRY(cudaMemsetAsync(p->d_labels, 0xff, sizeof(int32_t) * p->nodes, p->stream), "label reset");
    CUDA_TRY(cudaMemcpyAsync(p->d_mask, p->d_iso, sizeof(uint32_t) * p->mask_words, cudaMemcpyDeviceToDevice,
                             p->stream),
             "mask reset");
    CUDA_TRY(cudaStreamSynchronize(p->stream), "reset synchronize");
    p->needs_init = false;
    return B40C_SUCCESS;
}

int b40c_bfs_enact_limited(b40c_bfs_problem *p, int strategy, int mode, int32_t src, int32_t depth_limit,
                           int max_grid_size, const b40c_bfs_policy *policy)
{
    b40c::clear_error();
    if (!p) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null problem");
    if (src < 0 || src >= p->nodes) return b40c::fail(B40C_ERROR_INVALID_VALUE, "source %d out of range", src);
    if (max_grid_size < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "negative max_grid_size");
    b40c_bfs_policy pol;
    int rc = resolve_policy(strategy, policy, &pol);
    if (rc) return rc;
    // A caller that passes no policy at all (the reference's enactor calls)
    // gets 512-thread CTAs for the distance searches of the top-down
    // strategies: measured 2-10% faster than 256 threads on R-MAT 22, random
    // 2^21, grid2d-1000 and grid3d-256 (hybrid with its hand-off scaled to the
    // CTA size, enact_edge.cu).  Predecessor searches keep 256: their
    // warp-by-warp levels need CTAs of at most 256 threads.
    if (!policy && !p->mark_pred &&
        (strategy == B40C_EXPAND_CONTRACT || strategy == B40C_CONTRACT_EXPAND || strategy == B40C_TWO_PHASE ||
         strategy == B40C_HYBRID))
        pol.threads = 512;
    DeviceGuard guard(p->device);
    p->timed = false;
    switch (strategy) {
    case B40C_EXPAND_CONTRACT:
        rc = enact_vertex(p, mode, src, max_grid_size, pol, depth_limit, false);
        break;
    case B40C_DIRECTION_OPTIMIZING:
        if ((rc = check_symmetric(p))) break;
        rc = enact_vertex(p, mode, src, max_grid_size, pol, depth_limit, p->symmetric == 1);
        break;
    case B40C_CONTRACT_EXPAND:
    case B40C_TWO_PHASE:
    case B40C_HYBRID:
        rc = enact_edge(p, strategy, mode, src, max_grid_size, pol, depth_limit);
        break;
    default:
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "unknown strategy %d", strategy);
    }
    p->needs_init = true;
    return rc;
}

int b40c_bfs_enact(b40c_bfs_problem *p, int strategy, int mode, int32_t src, int max_grid_size,
                   const b40c_bfs_policy *policy)
{
    return b40c_bfs_enact_limited(p, strategy, mode, src, -1, max_grid_size, policy);
}

int b40c_bfs_stats(b40c_bfs_problem *p, int64_t *total_queued, int32_t *search_depth, double *avg_duty)
{
    b40c::clear_error();
    if (!p) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null problem");
    DeviceGuard guard(p->device);
    int rc = read_state(p);
    if (rc) return rc;
    if ((rc = check_state_errors(p))) return rc;
    if (total_queued) *total_queued = (int64_t)p->h_st->total_queued;
    if (search_depth) *search_depth = p->h_st->max_level + 1;
    if (avg_duty) {
        *avg_duty = 0.0;
        if (p->instrument) {
            unsigned long long d[4];
            CUDA_TRY(cudaMemcpy(d, p->d_duty, sizeof(d), cudaMemcpyDeviceToHost), "duty read");
            if (d[1]) *avg_duty = (double)d[0] / (double)d[1];
        }
    }
    return B40C_SUCCESS;
}

int b40c_bfs_problem_is_symmetric(b40c_bfs_problem *p, int *symmetric)
{
    b40c::clear_error();
    if (!p || !symmetric) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    DeviceGuard guard(p->device);
    int rc = check_symmetric(p);
    if (rc) return rc;
    *symmetric = p->symmetric;
    return B40C_SUCCESS;
}

int b40c_bfs_set_instrument(b40c_bfs_problem *p, int on)
{
    b40c::clear_error();
    if (!p) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null problem");
    DeviceGuard guard(p->device);
    if (on && !p->d_levels) {
        int rc;
        if ((rc = alloc_dev((void **)&p->d_levels, sizeof(LevelRecord) * kMaxLevelRecords, "level records"))) return rc;
        if ((rc = alloc_dev((void **)&p->d_duty, 4 * sizeof(unsigned long long), "duty counters"))) return rc;
        if ((rc = alloc_dev((void **)&p->d_arrive,
                            sizeof(unsigned long long) * kMaxArrivePasses * kMaxArriveCtas * kPhaseStamps,
                            "arrival times")))
            return rc;
    }
    p->instrument = on != 0;
    return B40C_SUCCESS;
}

int b40c_bfs_cta_arrivals(b40c_bfs_problem *p, uint64_t *out, int max_passes, int *ctas)
{
    b40c::clear_error();
    if (!p || !out || !ctas || max_passes < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "bad arguments");
    if (!p->instrument || !p->d_arrive)
        return b40c::fail(B40C_ERROR_NOT_READY, "instrumentation is off (b40c_bfs_set_instrument)");
    DeviceGuard guard(p->device);
    const int passes = std::min(max_passes, kMaxArrivePasses);
    const int g = std::min(p->last_grid, kMaxArriveCtas);
    std::vector<unsigned long long> h((size_t)kMaxArrivePasses * kMaxArriveCtas * kPhaseStamps);
    CUDA_TRY(cudaStreamSynchronize(p->stream), "stream synchronize");
    CUDA_TRY(cudaMemcpy(h.data(), p->d_arrive, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost),
             "arrival read");
    for (int k = 0; k < passes; k++)
        for (int c = 0; c < g; c++)
            for (int f = 0; f < kPhaseStamps; f++)
                out[((size_t)k * g + c) * kPhaseStamps + f] = h[((size_t)k * kMaxArriveCtas + c) * kPhaseStamps + f];
    *ctas = g;
    return B40C_SUCCESS;
}

int b40c_bfs_level_records(b40c_bfs_problem *p, b40c_level_record *out, int max_records, int *count)
{
    b40c::clear_error();
    if (!p || !out || !count || max_records < 0) return b40c::fail(B40C_ERROR_INVALID_VALUE, "bad arguments");
    if (!p->instrument) return b40c::fail(B40C_ERROR_NOT_READY, "instrumentation is off (b40c_bfs_set_instrument)");
    DeviceGuard guard(p->device);
    const int n = std::min(max_records, kMaxLevelRecords);
    std::vector<LevelRecord> h((size_t)std::max(n, 1));
    unsigned long long d[4];
    CUDA_TRY(cudaStreamSynchronize(p->stream), "stream synchronize");
    CUDA_TRY(cudaMemcpy(h.data(), p->d_levels, sizeof(LevelRecord) * n, cudaMemcpyDeviceToHost), "level records read");
    CUDA_TRY(cudaMemcpy(d, p->d_duty, sizeof(d), cudaMemcpyDeviceToHost), "duty read");
    int c = 0;
    while (c < n && h[c].t_ns != 0) {
        out[c].vertices = h[c].vertices;
        out[c].edges = h[c].edges;
        out[c].bottom_up = h[c].bottom_up;
        out[c].pass = h[c].pass;
        out[c].t_ns = h[c].t_ns;
        c++;
    }
    if (c < n) {  // closing record: when the last CTA finished
        out[c].vertices = out[c].edges = out[c].bottom_up = 0;
        out[c].pass = -1;
        out[c].t_ns = d[2];
        c++;
    }
    *count = c;
    return B40C_SUCCESS;
}

int b40c_bfs_last_elapsed_ms(b40c_bfs_problem *p, float *ms)
{
    b40c::clear_error();
    if (!p || !ms) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    if (!p->timed) return b40c::fail(B40C_ERROR_NOT_READY, "no timed search");
    DeviceGuard guard(p->device);
    CUDA_TRY(cudaEventSynchronize(p->ev1), "event synchronize");
    CUDA_TRY(cudaEventElapsedTime(ms, p->ev0, p->ev1), "event elapsed");
    return B40C_SUCCESS;
}

int b40c_bfs_recent_search_ms(b40c_bfs_problem *p, int count, float *out)
{
    b40c::clear_error();
    if (!p || !out || count < 1) return b40c::fail(B40C_ERROR_INVALID_VALUE, "bad arguments");
    if (count > p->ring_count)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "only %d timed searches recorded (ring of %d)", p->ring_count,
                          b40c_bfs_problem::kRing);
    DeviceGuard guard(p->device);
    const int R = b40c_bfs_problem::kRing;
    const int newest = (p->ring_pos + R - 1) % R;
    CUDA_TRY(cudaEventSynchronize(p->ring_b[newest]), "event synchronize");
    for (int i = 0; i < count; i++) {
        const int slot = (p->ring_pos + R - count + i) % R;
        CUDA_TRY(cudaEventElapsedTime(&out[i], p->ring_a[slot], p->ring_b[slot]), "event elapsed");
    }
    return B40C_SUCCESS;
}

int b40c_bfs_extract(b40c_bfs_problem *p, int32_t *h_labels)
{
    b40c::clear_error();
    if (!p || !h_labels) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    DeviceGuard guard(p->device);
    int rc = read_state(p);
    if (rc) return rc;
    if ((rc = check_state_errors(p))) return rc;
    CUDA_TRY(cudaMemcpyAsync(h_labels, p->d_labels, sizeof(int32_t) * p->nodes, cudaMemcpyDeviceToHost, p->stream),
             "label copy");
    CUDA_TRY(cudaStreamSynchronize(p->stream), "label copy synchronize");
    return B40C_SUCCESS;
}

int b40c_bfs_extract_wait(b40c_bfs_problem *p, int slot)
{
    b40c::clear_error();
    if (!p) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null problem");
    if (slot < 0 || slot > 1) return b40c::fail(B40C_ERROR_INVALID_VALUE, "staging slot %d (0 or 1)", slot);
    if (!p->stage_pending[slot]) return B40C_SUCCESS;
    DeviceGuard guard(p->device);
    p->stage_pending[slot] = false;
    CUDA_TRY(cudaEventSynchronize(p->landed_ev[slot]), "label copy synchronize");
    return error_status(p->h_stage_err[slot]);
}

int b40c_bfs_extract_async(b40c_bfs_problem *p, int32_t *h_labels, int slot)
{
    b40c::clear_error();
    if (!p || !h_labels) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    if (slot < 0 || slot > 1) return b40c::fail(B40C_ERROR_INVALID_VALUE, "staging slot %d (0 or 1)", slot);
    DeviceGuard guard(p->device);
    int rc;
    if (p->stage_pending[slot]) {
        // the slot's previous copy must land before its buffer is reused; its
        // status belonged to an earlier search and was not asked for
        p->stage_pending[slot] = false;
        CUDA_TRY(cudaEventSynchronize(p->landed_ev[slot]), "label copy synchronize");
    }
    if (!p->copy_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking), "copy stream");
        for (int i = 0; i < 2; i++) {
            CUDA_TRY(cudaEventCreateWithFlags(&p->staged_ev[i], cudaEventDisableTiming), "event");
            CUDA_TRY(cudaEventCreateWithFlags(&p->landed_ev[i], cudaEventDisableTiming), "event");
        }
        if ((rc = alloc_dev((void **)&p->d_stage_err, 8, "staging error words"))) return rc;
        CUDA_TRY(cudaHostAlloc((void **)&p->h_stage_err, 8, cudaHostAllocDefault), "pinned error words");
    }
    if (!p->d_stage[slot] &&
        (rc = alloc_dev((void **)&p->d_stage[slot], sizeof(int32_t) * std::max<int64_t>(p->nodes, 1), "label staging")))
        return rc;
    const int64_t n = p->nodes;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)p->sms * 8, (n / 4 + 255) / 256));
    stage_results_kernel<<<blocks, 256, 0, p->stream>>>(p->d_labels, p->d_stage[slot], n, &p->st->error,
                                                        p->d_stage_err + slot);
    CUDA_TRY(cudaGetLastError(), "staging launch");
    CUDA_TRY(cudaEventRecord(p->staged_ev[slot], p->stream), "event record");
    CUDA_TRY(cudaStreamWaitEvent(p->copy_stream, p->staged_ev[slot], 0), "stream wait");
    CUDA_TRY(cudaMemcpyAsync(h_labels, p->d_stage[slot], sizeof(int32_t) * n, cudaMemcpyDeviceToHost, p->copy_stream),
             "label copy");
    CUDA_TRY(cudaMemcpyAsync(p->h_stage_err + slot, p->d_stage_err + slot, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                             p->copy_stream),
             "error word copy");
    CUDA_TRY(cudaEventRecord(p->landed_ev[slot], p->copy_stream), "event record");
    p->stage_pending[slot] = true;
    return B40C_SUCCESS;
}

int b40c_bfs_device_view_get(b40c_bfs_problem *p, b40c_bfs_device_view *v)
{
    b40c::clear_error();
    if (!p || !v) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null argument");
    v->d_row_offsets = p->d_ro;
    v->d_column_indices = p->d_ci;
    v->d_labels = p->d_labels;
    v->d_visited_mask = p->d_mask;
    v->visited_mask_bytes = (p->nodes + 7) / 8;
    v->nodes = p->nodes;
    v->edges = p->edges;
    v->device = p->device;
    v->mark_predecessors = p->mark_pred;
    return B40C_SUCCESS;
}

}  // extern "C"
