// b40c_bfs_search_noalloc: a single-source BFS that allocates no memory.
//
// Who needs it: callers that must not (or cannot) allocate device memory at
// search time -- code running inside another framework's memory pool or a
// fixed memory budget, callers on a device whose memory is already fully
// reserved, and real-time paths where a cudaMalloc/cudaFree would stall or
// synchronise the device.  They pass the CSR and the label array as device
// pointers they already own; everything else the search needs (visited mask,
// the two vertex frontiers, the search state) lives in the fixed scratch
// array below, compiled into the library.
//
// The kernels are the library's expand-contract kernels (bfs_kernels.cuh),
// run as one persistent cooperative grid; only the storage differs.
#include <mutex>

#include "bfs_kernels.cuh"
#include "problem.h"

namespace b40c {
namespace noalloc {

constexpr int64_t kMaxNodes = 1 << 18;  // 262,144 vertices
constexpr int64_t kMaxEdges = 1 << 22;  // 4,194,304 directed edges
constexpr int kThreads = 256;

// Byte layout of the scratch array (every piece 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kStateBytes = align256(sizeof(SearchState));
constexpr size_t kMaskBytes = align256(sizeof(uint32_t) * ((kMaxNodes + 31) / 32));
constexpr size_t kVecBytes = align256(sizeof(int32_t) * (kMaxNodes + 1));
constexpr size_t kCfBytes = align256(sizeof(int32_t) * (kMaxEdges / dev::kChunkGrain + 2));
constexpr size_t kFrontierBytes = 3 * kVecBytes + kCfBytes;
constexpr size_t kScratchBytes = kStateBytes + kMaskBytes + 2 * kFrontierBytes;

// The scratch: one copy per device that loads the library, kept until the
// process exits.  In host code this name is only a host-side stand-in for the
// symbol; its device address comes from cudaGetSymbolAddress (set_up below).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Sets the search's source (the init kernel reads it from the state).
__global__ void seed_kernel(SearchState *st, int32_t src)
{
    st->src = src;
    st->depth_limit = -1;
}

struct DeviceSetup {
    unsigned char *scratch = nullptr;  // device address of g_scratch on this device
    int grid = 0;                      // co-resident CTAs of the expand-contract kernel
    int init_grid = 0;
};

constexpr int kMaxDevices = 64;
static DeviceSetup g_setup[kMaxDevices];
static std::mutex g_setup_mutex;

// Once per device, with that device current: the scratch's device address,
// the kernel's shared-memory attribute and its cooperative grid size.  These
// belong to the device's primary context: after a cudaDeviceReset in the same
// process they are stale, so the entry point must not be used after one.
static int set_up(int device, DeviceSetup **out)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup &d = g_setup[device];
    if (!d.scratch) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return b40c::fail((int)e, "cudaGetSymbolAddress of the search scratch failed: %s", cudaGetErrorString(e));
        }
        const void *kern = (const void *)dev::ec_kernel<kThreads, false, false>;
        const size_t smem = sizeof(dev::ExpandSmem<kThreads, false>);
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int per_sm = 0, sms = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess || per_sm < 1) {
            cudaGetLastError();
            return b40c::fail(e != cudaSuccess ? (int)e : B40C_ERROR_INVALID_CONFIGURATION,
                              "no-allocation search set-up failed: %s", cudaGetErrorString(e));
        }
        d.grid = per_sm * sms;
        d.init_grid = sms * 8;
        d.scratch = (unsigned char *)ptr;
    }
    *out = &d;
    return B40C_SUCCESS;
}

}  // namespace noalloc
}  // namespace b40c

using namespace b40c;

extern "C" int b40c_bfs_search_noalloc(const int32_t *d_row_offsets, const int32_t *d_column_indices, int64_t nodes,
                                       int64_t edges, int32_t src, int32_t *d_labels, void *cuda_stream)
{
    using namespace b40c::noalloc;
    b40c::clear_error();
    if (!d_row_offsets || (!d_column_indices && edges > 0) || !d_labels)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_bfs_search_noalloc: null device pointer");
    if (nodes <= 0 || edges < 0 || nodes > kMaxNodes || edges > kMaxEdges)
        return b40c::fail(B40C_ERROR_INVALID_VALUE,
                          "b40c_bfs_search_noalloc: graph of %lld vertices and %lld edges exceeds its fixed scratch "
                          "(at most %lld vertices and %lld edges); use b40c_bfs_problem_create instead",
                          (long long)nodes, (long long)edges, (long long)kMaxNodes, (long long)kMaxEdges);
    if (src < 0 || src >= nodes) return b40c::fail(B40C_ERROR_INVALID_VALUE, "source %d out of range", src);
    // int32 arrays: anything but a 4-byte aligned address would fault on the device
    if ((reinterpret_cast<uintptr_t>(d_row_offsets) | reinterpret_cast<uintptr_t>(d_column_indices) |
         reinterpret_cast<uintptr_t>(d_labels)) & 3u)
        return b40c::fail(B40C_ERROR_INVALID_VALUE, "b40c_bfs_search_noalloc: device arrays must be 4-byte aligned");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device >= kMaxDevices) {
        cudaGetLastError();
        return b40c::fail(B40C_ERROR_NO_DEVICE, "no usable current CUDA device");
    }
    DeviceSetup *d = nullptr;
    int rc = set_up(device, &d);
    if (rc) return rc;
    cudaStream_t stream = (cudaStream_t)cuda_stream;

    // carve the scratch; the init kernel below rewrites every piece the search reads
    unsigned char *base = d->scratch;
    SearchState *st = (SearchState *)base;
    base += kStateBytes;
    uint32_t *mask = (uint32_t *)base;
    base += kMaskBytes;
    BfsParams k{};
    for (int i = 0; i < 2; i++) {
        k.vf[i].v = (int32_t *)base;
        k.vf[i].col = (int32_t *)(base + kVecBytes);
        k.vf[i].P = (int32_t *)(base + 2 * kVecBytes);
        k.vf[i].cf = (int32_t *)(base + 3 * kVecBytes);
        base += kFrontierBytes;
    }
    k.row_offsets = d_row_offsets;
    k.column_indices = d_column_indices;
    k.labels = d_labels;
    k.mask = mask;
    k.nodes = (int32_t)nodes;
    k.edges = (int32_t)edges;
    k.mask_words = (int32_t)((nodes + 31) / 32);
    k.vcap = (int32_t)kMaxNodes;
    k.ecap = 0;
    k.max_chunks = 0;
    k.cf_cap = (int32_t)(kMaxEdges / dev::kChunkGrain + 2);
    k.slots = nullptr;
    k.st = st;
    k.max_levels = INT32_MAX;
    k.chunk_edges = dev::kChunkMax;
    k.warp_thresh = 32;
    k.cta_thresh = 512;
    k.warp_cull = 0;
    k.precheck = 1;
    k.saturation = 512;
    k.persistent = 1;
    k.skip_arrival_cta = -1;
    k.spin_limit = dev::kSpinLimit;
    k.bulk_ok = 1;  // device memory; the kernel aligns each bulk copy by address
    k.alloc_lookback = 0;  // one packed atomic per tile: no look-back slots needed
    k.direction_opt = 0;
    k.bu_alpha = 14;
    k.bu_beta = 24;
    k.small_edges = 1024;
    k.bu_scan = 1;
    k.bu_long = 256;
    k.hist_log = 0;
    k.bu_prefetch = 0;
    k.mask_alt = nullptr;  // never bottom-up
    k.hub2 = nullptr;
    k.levels = nullptr;
    k.duty = nullptr;
    k.cond_handle = 0;

    seed_kernel<<<1, 1, 0, stream>>>(st, src);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        dev::init_kernel<false, true, true><<<d->init_grid, kThreads, 0, stream>>>(k);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        void *args[] = {&k};
        e = cudaLaunchCooperativeKernel((const void *)dev::ec_kernel<kThreads, false, false>, dim3(d->grid), dim3(kThreads),
                                        args, sizeof(dev::ExpandSmem<kThreads, false>), stream);
    }
    // wait for the search and read its error word into a local variable
    unsigned error_word = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&error_word, &st->error, sizeof(error_word), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return b40c::fail((int)e, "no-allocation search failed: %s", cudaGetErrorString(e));
    }
    if (error_word & dev::kErrOverflow)
        return b40c::fail(B40C_ERROR_INVALID_CONFIGURATION, "no-allocation search: frontier overflow");
    if (error_word)
        return b40c::fail(B40C_ERROR_LAUNCH_TIMEOUT, "no-allocation search: a bounded device wait expired (0x%x)",
                          error_word);
    return B40C_SUCCESS;
}
