// COO -> CSR on the GPU: the conversion CsrGraph::FromCoo does on the host
// with a stable sort by row (csr_graph.cuh:109-152), as a stable LSD radix
// sort of the edges by row (8-bit digits, as many passes as the row ids need)
// plus a row histogram and scan for the offsets.  Within a row the edges keep
// their input order, so the result equals FromCoo's byte for byte.
//
// One radix pass over tiles of kTile edges:
//   upsweep   per-tile digit counts, stored digit-major (hist[d * tiles + t]);
//   scan      exclusive scan of hist: the first output slot of every
//             (digit, tile) run, tiles in input order;
//   scatter   every tile ranks its edges among equal digits in input order
//             (warp match + per-warp counts + a running count per digit) and
//             writes (row, col) to its run.
#include <algorithm>

#include "problem.h"

namespace b40c {
namespace coo {

constexpr int kThreads = 256;
constexpr int kPer = 8;
constexpr int kTile = kThreads * kPer;  // 2048 edges per tile
constexpr int kBins = 256;
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanThreads * kScanPer;

__device__ __forceinline__ unsigned lanemask_lt_u()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// count[r] = edges of row r; out-of-range ids set *bad and are not counted.
__global__ void row_count_kernel(const int32_t *rows, const int32_t *cols, int64_t m, int32_t n, int32_t *count,
                                 int32_t *bad)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const int32_t r = rows[i], c = cols[i];
        if ((uint32_t)r >= (uint32_t)n || (uint32_t)c >= (uint32_t)n) {
            *bad = 1;
            continue;
        }
        atomicAdd(count + r, 1);
    }
}

__global__ void upsweep_kernel(const int32_t *keys, int64_t m, int shift, int64_t tiles, int32_t *hist)
{
    __shared__ int h[kBins];
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        h[threadIdx.x] = 0;
        __syncthreads();
        const int64_t base = t * kTile;
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            const int64_t i = base + k * kThreads + threadIdx.x;
            if (i < m) atomicAdd(&h[(keys[i] >> shift) & (kBins - 1)], 1);
        }
        __syncthreads();
        hist[(int64_t)threadIdx.x * tiles + t] = h[threadIdx.x];
        __syncthreads();
    }
}

// Inclusive scan of one value per thread across a 1024-thread block; returns
// the inclusive prefix and leaves the block total in *total.
__device__ __forceinline__ int block_scan_inclusive(int x, int *warp_sums, int *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    const int r = x + (warp > 0 ? warp_sums[warp - 1] : 0);
    *total = warp_sums[31];
    __syncthreads();
    return r;
}

__global__ void scan_reduce_kernel(const int32_t *in, int64_t len, int32_t *block_sums)
{
    __shared__ int warp_sums[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPer;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++)
        if (base + k < len) s += in[base + k];
    int total;
    block_scan_inclusive(s, warp_sums, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// One block: exclusive scan of the block sums in place, chunk after chunk.
__global__ void scan_spine_kernel(int32_t *sums, int64_t count)
{
    __shared__ int warp_sums[32];
    int carry = 0;
    for (int64_t c0 = 0; c0 < count; c0 += kScanThreads) {
        const int64_t i = c0 + threadIdx.x;
        const int x = i < count ? sums[i] : 0;
        int total;
        const int inc = block_scan_inclusive(x, warp_sums, &total);
        if (i < count) sums[i] = carry + inc - x;
        carry += total;
    }
}

__global__ void scan_down_kernel(const int32_t *in, int64_t len, const int32_t *block_sums, int32_t *out)
{
    __shared__ int warp_sums[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPer;
    int v[kScanPer];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        v[k] = base + k < len ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int run = block_scan_inclusive(s, warp_sums, &total) - s + block_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        if (base + k < len) out[base + k] = run;
        run += v[k];
    }
}

__global__ void scatter_kernel(const int32_t *keys, const int32_t *vals, int64_t m, int shift, int64_t tiles,
                               const int32_t *offsets, int32_t *keys_out, int32_t *vals_out)
{
    __shared__ int running[kBins];
    __shared__ int wcnt[kThreads / 32][kBins];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        running[tid] = 0;
        const int64_t base = t * kTile;
        __syncthreads();
        for (int k = 0; k < kPer; k++) {
            const int64_t i = base + k * kThreads + tid;
            const bool valid = i < m;
            const int32_t key = valid ? keys[i] : 0;
            const int d = valid ? (key >> shift) & (kBins - 1) : -1 - lane;  // invalid lanes match nobody
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const int rank = __popc(peers & lanemask_lt_u());
#pragma unroll
            for (int j = 0; j < kBins / 32; j++) wcnt[warp][lane * (kBins / 32) + j] = 0;
            __syncwarp();
            if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
            __syncthreads();
            if (valid) {
                int pos = offsets[(int64_t)d * tiles + t] + running[d] + rank;
                for (int w = 0; w < warp; w++) pos += wcnt[w][d];
                if (keys_out) keys_out[pos] = key;  // the last pass needs no keys
                vals_out[pos] = vals[i];
            }
            __syncthreads();
            int add = 0;
#pragma unroll
            for (int w = 0; w < kThreads / 32; w++) add += wcnt[w][tid];
            running[tid] += add;
            __syncthreads();
        }
    }
}

}  // namespace coo

namespace rt {

namespace {

struct DeviceBuffer {
    void *p = nullptr;
    ~DeviceBuffer()
    {
        if (p) cudaFree(p);
    }
};

int exclusive_scan(int32_t *data, int64_t len, int32_t *sums, cudaStream_t s)
{
    using namespace coo;
    const int64_t blocks = (len + kScanTile - 1) / kScanTile;
    scan_reduce_kernel<<<(unsigned)blocks, kScanThreads, 0, s>>>(data, len, sums);
    scan_spine_kernel<<<1, kScanThreads, 0, s>>>(sums, blocks);
    scan_down_kernel<<<(unsigned)blocks, kScanThreads, 0, s>>>(data, len, sums, data);
    CUDA_TRY(cudaGetLastError(), "scan launch");
    return B40C_SUCCESS;
}

}  // namespace

// Stable by-row conversion of a device COO list into device CSR arrays
// (row_offsets[nodes + 1], column_indices[edges]); synchronous on `s`.
int coo_to_csr_device(const int32_t *d_rows, const int32_t *d_cols, int64_t nodes, int64_t edges, int32_t *d_ro,
                      int32_t *d_ci, cudaStream_t s, int sms)
{
    using namespace coo;
    const int64_t tiles = std::max<int64_t>((edges + kTile - 1) / kTile, 1);
    const int64_t hist_len = (int64_t)kBins * tiles;
    const int64_t scan_len = std::max<int64_t>(hist_len, nodes + 1);
    DeviceBuffer keys[2], vals[2], hist, sums, bad;
    int rc;
    if ((rc = alloc_dev(&hist.p, sizeof(int32_t) * hist_len, "radix histogram"))) return rc;
    if ((rc = alloc_dev(&sums.p, sizeof(int32_t) * ((scan_len + kScanTile - 1) / kScanTile + 1), "scan sums")))
        return rc;
    if ((rc = alloc_dev(&bad.p, sizeof(int32_t), "range flag"))) return rc;
    int32_t *h = (int32_t *)hist.p, *sm = (int32_t *)sums.p, *flag = (int32_t *)bad.p;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sms * 8));

    // row offsets: per-row counts, then an exclusive scan over nodes + 1 entries
    CUDA_TRY(cudaMemsetAsync(d_ro, 0, sizeof(int32_t) * (nodes + 1), s), "offset reset");
    CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int32_t), s), "flag reset");
    if (edges > 0) {
        row_count_kernel<<<grid, kThreads, 0, s>>>(d_rows, d_cols, edges, (int32_t)nodes, d_ro, flag);
        CUDA_TRY(cudaGetLastError(), "row count launch");
    }
    int32_t h_bad = 0;
    CUDA_TRY(cudaMemcpyAsync(&h_bad, flag, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "flag read");
    CUDA_TRY(cudaStreamSynchronize(s), "row count");
    if (h_bad) return b40c::fail(B40C_ERROR_INVALID_VALUE, "COO vertex id out of [0, %lld)", (long long)nodes);
    if ((rc = exclusive_scan(d_ro, nodes + 1, sm, s))) return rc;
    if (edges == 0) {
        CUDA_TRY(cudaStreamSynchronize(s), "scan");
        return B40C_SUCCESS;
    }

    // radix passes over the row ids' significant bits; pass p < last writes
    // buffer p & 1, the last pass writes only the column indices (into d_ci)
    int bits = 1;
    while (bits < 31 && ((int64_t)1 << bits) < nodes) bits++;
    const int passes = (bits + 7) / 8;
    for (int i = 0; i < 2 && i < passes - 1; i++) {
        if ((rc = alloc_dev(&keys[i].p, sizeof(int32_t) * edges, "radix keys"))) return rc;
        if ((rc = alloc_dev(&vals[i].p, sizeof(int32_t) * edges, "radix values"))) return rc;
    }
    const int32_t *kin = d_rows, *vin = d_cols;
    for (int pass = 0; pass < passes; pass++) {
        const bool last = pass == passes - 1;
        int32_t *kout = last ? nullptr : (int32_t *)keys[pass & 1].p;
        int32_t *vout = last ? d_ci : (int32_t *)vals[pass & 1].p;
        const int shift = 8 * pass;
        upsweep_kernel<<<grid, kThreads, 0, s>>>(kin, edges, shift, tiles, h);
        CUDA_TRY(cudaGetLastError(), "upsweep launch");
        if ((rc = exclusive_scan(h, hist_len, sm, s))) return rc;
        scatter_kernel<<<grid, kThreads, 0, s>>>(kin, vin, edges, shift, tiles, h, kout, vout);
        CUDA_TRY(cudaGetLastError(), "scatter launch");
        kin = kout;
        vin = vout;
    }
    CUDA_TRY(cudaStreamSynchronize(s), "radix sort");
    return B40C_SUCCESS;
}

}  // namespace rt
}  // namespace b40c

using namespace b40c;
using namespace b40c::rt;

extern "C" {

int b40c_coo_to_csr_device(const int32_t *d_rows, const int32_t *d_cols, int64_t nodes, int64_t edges,
                           int32_t *d_row_offsets, int32_t *d_column_indices, void *cuda_stream)
{
    b40c::clear_error();
    if (((!d_rows || !d_cols || !d_column_indices) && edges > 0) || !d_row_offsets || nodes <= 0 || edges < 0 ||
        nodes >= INT32_MAX || edges >= INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_coo_to_csr_device: bad arguments");
    int device = 0, sms = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return b40c::fail(B40C_ERROR_NO_DEVICE, "no usable current CUDA device");
    }
    return coo_to_csr_device(d_rows, d_cols, nodes, edges, d_row_offsets, d_column_indices,
                             (cudaStream_t)cuda_stream, sms);
}

int b40c_bfs_problem_create_coo(const int32_t *h_rows, const int32_t *h_cols, int64_t nodes, int64_t edges,
                                int mark_predecessors, int device, b40c_bfs_problem **out)
{
    b40c::clear_error();
    if (!out) return b40c::fail(B40C_ERROR_INVALID_VALUE, "null output handle");
    *out = nullptr;
    if ((!h_rows || !h_cols) && edges > 0)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "null COO arrays");
    if (nodes <= 0 || edges < 0 || nodes >= (int64_t)1 << 30 || edges >= (int64_t)INT32_MAX)
        return b40c::fail(B40C_ERROR_INVALID_VALUE,
                          "invalid COO (nodes %lld, edges %lld; need 0 < nodes < 2^30, edges < 2^31)",
                          (long long)nodes, (long long)edges);
    auto load = [&](b40c_bfs_problem *p) -> int {
        int rc;
        if ((rc = alloc_dev((void **)&p->d_ro, sizeof(int32_t) * (nodes + 1), "row offsets"))) return rc;
        if ((rc = alloc_dev((void **)&p->d_ci, sizeof(int32_t) * std::max<int64_t>(edges, 1), "column indices")))
            return rc;
        DeviceBuffer rows, cols;
        const size_t bytes = sizeof(int32_t) * (size_t)std::max<int64_t>(edges, 1);
        if ((rc = alloc_dev(&rows.p, bytes, "COO rows"))) return rc;
        if ((rc = alloc_dev(&cols.p, bytes, "COO columns"))) return rc;
        if (edges > 0) {
            CUDA_TRY(cudaMemcpyAsync(rows.p, h_rows, bytes, cudaMemcpyHostToDevice, p->stream), "COO upload");
            CUDA_TRY(cudaMemcpyAsync(cols.p, h_cols, bytes, cudaMemcpyHostToDevice, p->stream), "COO upload");
        }
        return coo_to_csr_device((const int32_t *)rows.p, (const int32_t *)cols.p, nodes, edges, p->d_ro, p->d_ci,
                                 p->stream, p->sms);
    };
    return create_problem(nodes, edges, mark_predecessors, 0, device, load, out);
}

}  // extern "C"
