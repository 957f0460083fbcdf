// Device-resident search state and the kernel parameter block shared by the
// host runtime (bfs_runtime.cu) and the kernels (bfs_kernels.cuh).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace b40c {

namespace dev {
struct LookbackSlot;
}

// One vertex frontier: for entry i, `v[i]` is the vertex, `col[i]` the start of
// its adjacency list and `P[i]` the exclusive prefix of the degrees of
// entries 0..i-1 (so entry i owns edges [P[i], P[i+1]) of the level's
// flattened edge space).  P has capacity + 1 slots.  Only vertices with at
// least one edge are enqueued.
struct VertexFrontier {
    int32_t *v;
    int32_t *col;
    int32_t *P;
    int32_t *cf;  // chunk-first index: cf[c] = entry owning edge c * kChunkGrain of the flattened edge space
};

// One edge frontier: neighbour ids (and their predecessors when marking
// predecessors), duplicates allowed.
struct EdgeFrontier {
    int32_t *v;
    int32_t *pred;
};

// Rotating/ping-pong counters written by the kernels (the role of the
// reference's CtaWorkProgress, util/cta_work_progress.cuh:69-223).
struct alignas(128) SearchState {
    // ---- line 0: frontier counters, updated by every CTA (one atomic per tile)
    // Frontier sizes, rotating over passes (a pass is one level of
    // expand-contract, or one phase of a level of the edge strategies):
    // pass k reads qe[k % 3] and accumulates its output frontier into
    // qe[(k + 1) % 3]; each value packs (count << 32 | edge total).
    unsigned long long qe[3];
    uint32_t tile_ctr[3];      // look-back tile counters, by pass % 3
    // bottom-up list mode (direction-optimizing distance searches): the list of
    // still-unvisited vertices a pass reads, by pass % 3 like qe: buffer index
    // (-1: none yet) and entries
    int32_t ul_sel[3];
    uint32_t ul_count[3];
    // ---- line 1: the grid barrier's arrival counter (polled by waiting CTAs)
    alignas(128) unsigned long long barrier;  // arrivals of the current persistent launch
    // ---- line 2: the error word (polled now and then) and launch epilogue counter
    alignas(128) uint32_t error;  // dev::kErr* bits
    uint32_t finished;            // CTAs that finished the current non-persistent launch
    // ---- line 3 on: per-search bookkeeping
    alignas(128) int32_t cur_level;  // next level to process
    unsigned long long epoch;  // look-back epoch base for this search
    int32_t max_level;         // deepest level at which a vertex was labelled
    int32_t done;              // 1 once the frontier emptied (or the depth limit was hit)
    int32_t saturated;         // 1 when a hybrid fused launch handed off
    unsigned long long total_queued;  // sum of processed frontier lengths
    int32_t src;               // source vertex (read by the init kernel)
    int32_t depth_limit;       // < 0: unlimited
    // direction-optimizing bookkeeping, rotating like qe: pass k reads [k % 3]
    // and block 0 writes [(k + 1) % 3]
    int32_t dir[3];            // 1: the previous level ran bottom-up, 2: bottom-up with its frontier deferred
    int32_t mask_sel[3];       // which visited-mask buffer holds the visited set (0: mask, 1: mask_alt)
    unsigned long long visited_edges[3];  // degree sum of the vertices visited before the pass
    // level at which a persistent launch resumes after a small-frontier phase of
    // CTA 0, by phase parity (a slot is rewritten only two phases later, after
    // every CTA has read it)
    int32_t solo_resume[2];
    // the same for a phase of mid-size top-down levels run by the first
    // kSubgridCtas CTAs alone
    int32_t sub_resume[2];
    // slots of a deferred bottom-up frontier built at the start of the next
    // level (count << 32 | edge total; cleared when the bottom-up level starts)
    unsigned long long mat_ctr;
    // arrival counter of the barrier among the CTAs of a sub-grid phase (its own line)
    alignas(128) unsigned long long sub_barrier;
};

__host__ __device__ inline int qe_count(unsigned long long x) { return (int)(x >> 32); }
__host__ __device__ inline int qe_edges(unsigned long long x) { return (int)(x & 0xffffffffull); }
__host__ __device__ inline int pass_of(int level, int phase, bool edge_strategy)
{
    return edge_strategy ? 2 * level + phase : level;
}

// Per-level record written when a search is instrumented (the role of the
// reference's KernelRuntimeStats, util/kernel_runtime_stats.cuh:45-126, and of
// its driver's per-level histogram, test/bfs/test_bfs.cu:264-337).
struct LevelRecord {
    int32_t vertices;          // frontier entries (vertex frontier) or items (edge frontier) of the pass
    int32_t edges;             // edges of the vertex frontier (0 for edge-frontier passes)
    int32_t bottom_up;         // 1 when the level ran bottom-up
    int32_t pass;
    unsigned long long t_ns;   // %globaltimer when block 0 started the pass
};
constexpr int kMaxLevelRecords = 1 << 16;
// Per-CTA times (%globaltimer ns) for the first kMaxArrivePasses passes of an
// instrumented persistent search: [pass][cta][kPhaseStamps], phases 0..5
// mark steps of the CTA's first work chunk of the level (see stamp sites),
// phase kPhaseArrive its arrival at the end-of-level grid barrier.
constexpr int kMaxArrivePasses = 64;
constexpr int kMaxArriveCtas = 2048;
constexpr int kPhaseStamps = 8;
constexpr int kPhaseArrive = 7;

// Sources added to a batched search while it runs (b40c_msbfs_join): the
// host copies request j into src/slot/limit[j] and then raises `count`; at
// the end of each level block 0 takes the requests up to count, seeds them as
// sources of the next level and sets `taken`.  A slot's labels count from the
// level it was seeded at, so they are the distances of a search from that
// source alone.  Device memory, reset by the batch's seed kernel.
struct MsJoin {
    int32_t count;              // requests written by the host
    int32_t taken;              // requests the search has taken (block 0)
    unsigned long long used;    // slots in use: the batch's k plus the joined ones
    int32_t src[64], slot[64], limit[64];
};

// Kernel parameter block.
struct BfsParams {
    const int32_t *row_offsets;
    const int32_t *column_indices;
    int32_t *labels;
    uint32_t *mask;
    int32_t nodes;
    int32_t edges;
    int32_t mask_words;
    int32_t vcap;  // vertex frontier capacity (entries)
    int32_t ecap;  // edge frontier capacity (entries)
    int32_t max_chunks;
    int32_t cf_cap;  // entries of each vertex frontier's cf array (a level's edge total / kChunkGrain + 2)
    VertexFrontier vf[2];
    EdgeFrontier ef[2];
    dev::LookbackSlot *slots;
    SearchState *st;
    int32_t max_levels;       // levels this launch may process (1 = one level per launch)
    int32_t chunk_edges;      // C_max for this launch (<= kChunkMax)
    int32_t warp_thresh;
    int32_t cta_thresh;
    int32_t warp_cull;
    int32_t precheck;
    int32_t saturation;       // hybrid: leave the fused kernel when items > gridDim * saturation
    int32_t persistent;       // 1: loop over levels with the grid barrier
    int32_t skip_arrival_cta; // test-only fault injection: this CTA never arrives (-1 = off)
    uint32_t late_start_ns;   // test-only: CTAs other than 0 of a persistent launch start this late (0 = off)
    uint32_t spin_limit;      // polls before a device-side wait gives up (dev::kSpinLimit; tests pass less)
    int32_t bulk_ok;          // 1: a sub-round inside one adjacency list may be staged by cp.async.bulk
                              // (column_indices is device memory; 0 for a host-mapped CSR)
    int32_t edge_pingpong;    // edge strategies: 1 = two edge frontiers (EDGE_FRONTIERS), 0 = one (MIXED)
    int32_t phase_mask;       // edge kernel: 1 = contract, 2 = expand, 3 = both per level (persistent)
    int32_t hybrid;           // edge kernel: leave the persistent loop when the frontier saturates
    int32_t alloc_lookback;   // 1: frontier slots by decoupled look-back, 0: one atomic per tile
    int32_t direction_opt;    // 1: levels may run bottom-up (symmetric graphs only)
    int32_t bu_alpha;         // switch to bottom-up when frontier edges > unvisited edges / alpha
    int32_t bu_beta;          // switch back to top-down when frontier vertices < n / beta
    int32_t small_edges;      // persistent launches: frontiers with at most this many edges run on CTA 0 alone
    int32_t subgrid_edges;    // persistent launches: top-down frontiers with more than small_edges and at most
                              // this many edges run on the first kSubgridCtas CTAs alone (0: off)
    int32_t bu_scan;          // bottom-up continuation: 1 per lane, 2 per CTA (edge-parallel worklist)
    int32_t bu_long;          // bottom-up: lists longer than this are searched by the whole warp
    int32_t hist_log;         // history cull table of 2^hist_log entries per CTA (0: off)
    int32_t bu_prefetch;      // 1: the first bottom-up level stages each next chunk with bulk copies
    int32_t warp_contract;    // 1: contract passes run warp by warp (no CTA barriers), 0: CTA sub-rounds
    int32_t warp_bu;          // 1: first bottom-up levels of counting runs go warp by warp
    int32_t bu_defer;         // persistent bottom-up levels count their discoveries; the frontier is built
                              // from the mask buffers only when a top-down level follows
    const uint32_t *iso;      // bit v: v has no edges in or out; a search starts with these bits visited (null: none)
    const int2 *hub2;         // per vertex its two highest-degree neighbours, probed first bottom-up (null: off)
    int32_t *ul[2];           // unvisited-vertex lists of bottom-up list mode (null: off; distance mode only)
    uint32_t *mask_alt;       // second visited-mask buffer: a bottom-up level reads one buffer and writes
                              // every word of the other (old bits | its discoveries), then they swap
    LevelRecord *levels;      // per-pass records when instrumented, else null
    unsigned long long *duty; // [0] sum over CTAs of busy ns, [1] sum of lifetime ns (instrumented)
    unsigned long long *arrive;  // [pass][cta] %globaltimer at the end-of-level barrier (instrumented)
    unsigned long long cond_handle;  // cudaGraphConditionalHandle (graph mode), 0 = none
    // 1: the init kernel takes the source and depth limit from src_arg /
    // depth_arg (and stores them in the state); 0: they were copied into the
    // state before it runs (CUDA-graph replays re-point that copy per launch)
    int32_t src_by_value;
    int32_t src_arg, depth_arg;
};

}  // namespace b40c
