// Host-side state of a BFS problem (the role of bfs::CsrProblem and the
// enactors' lazily allocated resources) shared by the runtime translation
// units: problem.cu (C ABI, allocation), enact_vertex.cu (expand-contract),
// enact_edge.cu (contract-expand, two-phase, hybrid).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>

#include "b40c_bfs.h"
#include "bfs_state.h"
#include "device_primitives.cuh"
#include "errors.h"

#define CUDA_TRY(call, what)                                                                             \
    do {                                                                                                 \
        cudaError_t _e = (call);                                                                         \
        if (_e != cudaSuccess) {                                                                         \
            cudaGetLastError();                                                                          \
            return b40c::fail((int)_e, "%s failed: %s", what, cudaGetErrorString(_e));                  \
        }                                                                                                \
    } while (0)


struct b40c_bfs_problem {
    int device = 0;
    int64_t nodes = 0, edges = 0;
    int mark_pred = 0;
    int stream_from_host = 0;
    int sms = 0;
    // CSR
    int32_t *d_ro = nullptr, *d_ci = nullptr;
    bool own_csr = true;
    const void *reg_ro = nullptr, *reg_ci = nullptr;  // host arrays registered for zero-copy
    // search arrays
    int32_t *d_labels = nullptr;
    uint32_t *d_mask = nullptr;
    uint32_t *d_next = nullptr;  // second visited-mask buffer (bottom-up levels write it whole)
    uint32_t *d_iso = nullptr;   // bit v: vertex v has no edges in or out (pre-set in every search's visited mask)
    int32_t *d_hub2 = nullptr;   // [2n] per vertex its two highest-degree neighbours (symmetric graphs, lazily)
    int32_t *d_ul[2] = {nullptr, nullptr};  // [n] each: bottom-up unvisited lists (distance searches, lazily)
    int32_t mask_words = 0;
    int symmetric = -1;          // -1 unknown, else the cached result of the device symmetry test
    // batched multi-source searches (allocated on first use)
    unsigned long long *d_ms_visited = nullptr, *d_ms_fmask[2] = {nullptr, nullptr};
    int32_t *d_ms_labels = nullptr;
    int32_t ms_labels_k = 0;       // sources the label array is sized for
    int32_t *d_ms_src = nullptr;   // [64] depth limit of each source slot
    int32_t *d_ms_depth = nullptr; // [64] search depth of each source slot
    int32_t *d_ms_off = nullptr;   // [64] level at which each slot's source was seeded
    int32_t ms_k = 0;              // sources of the last batch
    // sources joining the batch in flight (b40c_msbfs_join): the device request
    // block, its pinned host staging, the stream the requests are copied on and
    // the event after which they may be (the batch's seed kernel)
    b40c::MsJoin *d_ms_join = nullptr, *h_ms_join = nullptr;
    int32_t *h_ms_seq = nullptr;   // pinned 0..64: request counts copied from here (never rewritten)
    cudaStream_t join_stream = nullptr;
    cudaEvent_t ms_seeded_ev = nullptr;
    int32_t ms_joins = 0;          // requests sent to the batch in flight
    // instrumentation (per-pass records, CTA duty)
    bool instrument = false;
    b40c::LevelRecord *d_levels = nullptr;
    unsigned long long *d_duty = nullptr;
    unsigned long long *d_arrive = nullptr;  // [kMaxArrivePasses][kMaxArriveCtas]
    int last_grid = 0;                       // CTAs of the last persistent launch
    // frontiers
    b40c::VertexFrontier vf[2] = {};
    int64_t vcap[2] = {0, 0};
    b40c::EdgeFrontier ef[2] = {};
    int64_t ecap[2] = {0, 0};
    double queue_sizing = 1.3;
    b40c::dev::LookbackSlot *slots = nullptr;
    int32_t max_slots = 0;
    b40c::SearchState *st = nullptr;
    b40c::SearchState *h_st = nullptr;  // pinned mirror
    // pinned (source, depth limit) of each enact, one pair per timing-ring slot:
    // an enact's upload reads its own pair, so enacts queued back to back
    // never see a later call's source
    int32_t *h_src_ring = nullptr;
    // streams / timing
    cudaStream_t stream = nullptr, own_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // ring of event pairs bracketing the search kernels (after source set-up)
    // of the most recent enacts, for per-launch device times
    static constexpr int kRing = 256;
    cudaEvent_t ring_a[kRing] = {}, ring_b[kRing] = {};
    int ring_pos = 0, ring_count = 0;
    bool timed = false;
    bool needs_init = true;  // labels/mask dirty since the last reset
    // CUDA graphs of whole searches (ENACT_GRAPH), one per strategy, rebuilt
    // when the kernel parameters (buffers, policy) or the grid change
    cudaGraphExec_t graph_exec[5] = {};
    cudaGraph_t graph_def[5] = {};           // kept for re-pointing the source copy per launch
    cudaGraphNode_t graph_copy_node[5] = {};  // the source-upload memcpy node of each graph
    b40c::BfsParams graph_params[5] = {};
    int graph_grid[5] = {};
    // pipelined read-back (b40c_bfs_extract_async): two device staging slots,
    // each with the search's error word, copied to the host on copy_stream
    int32_t *d_stage[2] = {};
    uint32_t *d_stage_err = nullptr;  // [2]
    uint32_t *h_stage_err = nullptr;  // [2], pinned
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t staged_ev[2] = {}, landed_ev[2] = {};
    bool stage_pending[2] = {};
};

namespace b40c {
namespace rt {

constexpr int kThreads = 256;
constexpr int kHistLog = 12;  // history cull table: 4096 vertex ids (16 KB) per CTA

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// The pinned (source, depth limit) pair of the enact being issued.
inline const int32_t *source_slot(const b40c_bfs_problem *p) { return p->h_src_ring + 2 * p->ring_pos; }

int alloc_dev(void **p, size_t bytes, const char *what);
void free_vf(VertexFrontier &f);
void free_ef(EdgeFrontier &f);
int ensure_vf(b40c_bfs_problem *p, int i, int64_t cap);
int ensure_ef(b40c_bfs_problem *p, int i, int64_t cap);
int64_t cap_of(double qs, int64_t base);
int64_t device_bytes(const b40c_bfs_problem *p);
// A problem handle whose CSR arrays `load` fills (upload, zero-copy mapping or
// a device-side build); everything else is allocated here.
int create_problem(int64_t nodes, int64_t edges, int mark_pred, int stream_from_host, int device,
                   const std::function<int(b40c_bfs_problem *)> &load, b40c_bfs_problem **out);
int64_t planned_bytes(int64_t n, int64_t m, int k, double qs);
int ensure_slots(b40c_bfs_problem *p);
BfsParams make_params(b40c_bfs_problem *p, const b40c_bfs_policy &pol);
uint32_t test_spin_limit();
b40c_bfs_policy default_policy(int strategy);
int resolve_policy(int strategy, const b40c_bfs_policy *in, b40c_bfs_policy *out);
int read_state(b40c_bfs_problem *p);
int check_state_errors(b40c_bfs_problem *p);
int persistent_grid(b40c_bfs_problem *p, const void *kernel, const b40c_bfs_policy &pol, int max_grid, size_t smem,
                    int *grid);
int finish_timing(b40c_bfs_problem *p);
int begin_instrumented(b40c_bfs_problem *p);
void free_graphs(b40c_bfs_problem *p);

// One kernel launch of a captured search.
struct KernelNode {
    const void *func;
    dim3 grid, block;
    size_t smem;
    BfsParams params;
};
// Builds (or reuses) and launches the whole-search graph of `slot`: source
// upload -> `init` -> conditional WHILE { body[0..n_body) }.  The body's
// last node sets the loop condition (its params get the handle).
int run_graph(b40c_bfs_problem *p, int slot, const KernelNode &init, KernelNode *body, int n_body);

// enactors
int enact_vertex(b40c_bfs_problem *p, int mode, int32_t src, int max_grid, const b40c_bfs_policy &pol,
                 int32_t depth_limit, bool direction_optimizing);
int check_symmetric(b40c_bfs_problem *p);
int ensure_hubs(b40c_bfs_problem *p);
int ensure_unvisited_lists(b40c_bfs_problem *p);
void free_batch(b40c_bfs_problem *p);
int ensure_batch(b40c_bfs_problem *p, int k);
// Queues a batched search of k <= 64 sources on p->stream (asynchronous).
int enact_batch(b40c_bfs_problem *p, const int32_t *sources, const int32_t *limits, int k, int max_grid,
                const b40c_bfs_policy &pol);
int enact_edge(b40c_bfs_problem *p, int strategy, int mode, int32_t src, int max_grid, const b40c_bfs_policy &pol,
               int32_t depth_limit);

}  // namespace rt
}  // namespace b40c
