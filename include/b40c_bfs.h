/*
 * b40c_bfs.h — C-ABI boundary of the B200-native single-GPU BFS library
 * (libb40c_bfs.so).  Plain pointers and sizes only; no CUDA or torch types.
 *
 * The reference (b40c, "Back40Computing" v1.0.1042) exposes this path as a
 * header-only C++ template API; its C++ callers keep that API through the
 * shims under include/b40c/, which forward to the entry points below.  Each
 * entry point names the reference interface it replaces (file:line in the
 * reference tree).
 *
 * Conventions
 *  - Every function returns an int status whose values are the cudaError_t
 *    values the reference returns for the same condition (0 = success).
 *    b40c_last_error_string() describes the last failure of the calling
 *    thread.
 *  - The caller owns host buffers; a problem handle owns its device buffers.
 *  - A handle is used by one host thread at a time; its work is ordered on
 *    the handle's CUDA stream (b40c_bfs_set_stream), default: a stream the
 *    handle creates.
 *  - Vertex ids, row offsets and labels are int32 on the device (the
 *    reference driver's graphs use SizeT = int; its one 64-bit VertexId graph
 *    type, "g500", is narrowed to int32 ids by the C++ CsrProblem).
 *  - b40c_bfs_policy grows at its end between versions: callers pass the
 *    struct of the header they were built with, so rebuild against this
 *    header (a caller built against an older one passes a shorter struct).
 */
#ifndef B40C_BFS_H
#define B40C_BFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (numerically equal to cudaError_t) -------------------- */
#define B40C_SUCCESS                        0
#define B40C_ERROR_INVALID_VALUE            1    /* cudaErrorInvalidValue */
#define B40C_ERROR_MEMORY_ALLOCATION        2    /* cudaErrorMemoryAllocation */
#define B40C_ERROR_INVALID_CONFIGURATION    9    /* cudaErrorInvalidConfiguration: frontier queue overflow
                                                    (enactor_contract_expand.cuh:319-324) */
#define B40C_ERROR_INVALID_DEVICE_FUNCTION  98   /* cudaErrorInvalidDeviceFunction: no kernel for this device */
#define B40C_ERROR_NO_DEVICE                100  /* cudaErrorNoDevice */
#define B40C_ERROR_NOT_READY                600  /* cudaErrorNotReady */
#define B40C_ERROR_LAUNCH_TIMEOUT           702  /* cudaErrorLaunchTimeout: a bounded device-side wait expired */
#define B40C_ERROR_NOT_SUPPORTED            801  /* cudaErrorNotSupported */
#define B40C_ERROR_INTERNAL                 999  /* cudaErrorUnknown: a device-side consistency check failed */

/* ---- enums ---------------------------------------------------------------- */

/* bfs::FrontierType, csr_problem.cuh:54-61 */
enum {
    B40C_VERTEX_FRONTIERS = 0,   /* two O(n) vertex frontiers */
    B40C_EDGE_FRONTIERS = 1,     /* two O(m) edge frontiers */
    B40C_MIXED_FRONTIERS = 2,    /* one O(n) vertex frontier, one O(m) edge frontier */
    B40C_MULTI_GPU_FRONTIERS = 3 /* accepted for API compatibility; treated as MIXED (single GPU only) */
};

/* Strategy, test/bfs/test_bfs.cu:72-79 (same numbering) */
enum {
    B40C_EXPAND_CONTRACT = 0, /* EnactorExpandContract   (enactor_expand_contract.cuh:59) */
    B40C_CONTRACT_EXPAND = 1, /* EnactorContractExpand   (enactor_contract_expand.cuh:61) */
    B40C_TWO_PHASE = 2,       /* EnactorTwoPhase         (enactor_two_phase.cuh:68) */
    B40C_HYBRID = 3,          /* EnactorHybrid           (enactor_hybrid.cuh:64) */
    B40C_DIRECTION_OPTIMIZING = 4 /* no counterpart in the reference: expand-contract top-down levels plus
                                     bottom-up levels while the frontier is large (undirected graphs;
                                     the same labels; plain expand-contract on a directed graph) */
};

/* How the levels of one search are launched. */
enum {
    B40C_ENACT_FUSED = 0,     /* EnactFusedSearch: one persistent grid, bounded software barrier between levels */
    B40C_ENACT_ITERATIVE = 1, /* EnactIterativeSearch: one launch per level, host reads the frontier size */
    B40C_ENACT_GRAPH = 2      /* whole search replayed as one CUDA graph (conditional WHILE node over levels) */
};

/* Runtime kernel policy (replaces the reference's compile-time KernelPolicy
 * template parameters, e.g. enactor_contract_expand.cuh:339-373).  A zero
 * field means "use the tuned default". */
typedef struct b40c_bfs_policy {
    int32_t threads;               /* CTA size: 128, 256 or 512 (default 256; b40c_bfs_enact with no policy
                                      at all runs 512 for the distance searches of expand-contract,
                                      contract-expand, two-phase and hybrid) */
    int32_t ctas_per_sm;           /* resident CTAs per SM for persistent grids (0 = occupancy limit) */
    int32_t chunk_edges;           /* edges (or edge-frontier items) per sub-round of a CTA's share of a level:
                                      a multiple of 32 in [256, 2048] (default 2048) */
    int32_t warp_gather_threshold; /* run length at or above which a warp gathers cooperatively (>= 32) */
    int32_t cta_gather_threshold;  /* run length at or above which the CTA gathers with bulk staging */
    int32_t saturation_quit;       /* hybrid: queue items per CTA of 256 threads (scaled for other CTA sizes)
                                      above which the search leaves the fused kernel */
    int32_t warp_cull;             /* 1: drop duplicate neighbours within a warp before the bitmask test,
                                      -1: do not (default) */
    int32_t bitmask_precheck;      /* 1: read the visited word (through L1) before the atomic test-and-set
                                      (default), 2: read it from L2 (never stale), -1: go straight to the
                                      atomic (default of direction-optimizing) */
    int32_t queue_allocation;      /* frontier-slot allocation per tile of output: 1 = decoupled look-back
                                      over tile ids, 2 = one packed 64-bit atomicAdd; 0 = default */
    int32_t bottom_up_alpha;       /* direction-optimizing: go bottom-up when frontier edges exceed
                                      unvisited edges / alpha */
    int32_t bottom_up_beta;        /* direction-optimizing: return top-down when the frontier holds fewer
                                      than nodes / beta vertices */
    int32_t small_frontier_edges;  /* fused searches: runs of levels whose frontier has at most this many
                                      edges are processed by one CTA alone (CTA-level barriers only);
                                      -1 disables */
    int32_t bottom_up_scan;        /* bottom-up levels, vertices whose first probes found no parent:
                                      1 = each lane scans its own list on (lists longer than 256 by the
                                      whole warp); the only variant built (CTA-wide edge-parallel scans
                                      measured slower); 0 = default */
    int32_t bottom_up_hub_probes;  /* bottom-up levels and batched pull levels first probe
                                      each vertex's two highest-degree neighbours (a per-vertex pair
                                      built once per symmetric problem, 8 bytes per vertex):
                                      1 = on (default), -1 = off */
    int32_t bottom_up_list;        /* distance searches: the first bottom-up level lists the vertices it
                                      left unvisited and later bottom-up levels scan only that list
                                      (testing neighbours on the labels; a kernel variant of its own):
                                      1 = on, -1 = off (default: measured slower overall on R-MAT and
                                      uniform graphs) */
    int32_t bottom_up_defer_frontier; /* fused direction-optimizing searches: a bottom-up level only counts
                                      its discoveries (and their edges); their vertex frontier is built
                                      from the two visited-mask buffers only when a top-down level
                                      follows: 1 = on (default), -1 = off */
    int32_t subgrid_frontier_edges; /* fused searches: runs of top-down levels with more than
                                      small_frontier_edges and at most this many edges run on 16 CTAs
                                      with a barrier of their own while the rest of the grid waits (the
                                      mid-size levels of high-diameter graphs); -1 = off (default) */
    int32_t bottom_up_long_list;   /* bottom-up levels: a vertex whose list is longer than this (and whose
                                      first probes found no parent) is searched by its whole warp, 32
                                      neighbours at a time; shorter lists are scanned by one lane, four at
                                      a time (>= 4; 0 = default 256) */
    int32_t history_cull;          /* top-down levels and contractions: each CTA remembers, in a 4096-entry
                                      shared-memory table, the neighbours it has already sent to the
                                      visited test and drops repeats without touching the visited mask
                                      (the reference's history culling): 1 = on, -1 = off (default) */
    int32_t bottom_up_prefetch;    /* the first bottom-up level of a run stages each next chunk's visited words,
                                      row offsets and hub pairs into shared memory with bulk copies while it
                                      scans the current one (25 KB of shared memory per CTA): 1 = on, -1 = off;
                                      default: on for 512-thread CTAs whose first bottom-up levels run in
                                      CTA-wide chunks (warp_bottom_up = -1), else off */
    int32_t warp_contract;         /* levels with at least a full 2048-edge sub-round per CTA, warp by warp:
                                      the contract and expand passes of the edge-frontier strategies
                                      (contract-expand, two-phase, hybrid), the top-down levels of
                                      expand-contract and direction-optimizing searches (predecessor
                                      searches: CTAs of up to 256 threads), and the pull levels of
                                      batched searches.  1 = each warp works through its own slices of
                                      the level, dealt over every warp of the grid, with no CTA barriers,
                                      and sends its winners to the vertex frontier in flushes of its own
                                      (one packed atomic each; default), -1 = CTA-wide sub-rounds
                                      (queue_allocation applies) */
    int32_t warp_bottom_up;        /* direction-optimizing fused searches, the first bottom-up level of a
                                      run when it only counts its discoveries: 1 = each warp takes blocks
                                      of vertex ids dealt over every warp of the grid, with no CTA
                                      barriers (default; bottom_up_prefetch does not apply), -1 = CTA-wide
                                      chunks */
} b40c_bfs_policy;

typedef struct b40c_bfs_problem b40c_bfs_problem; /* opaque */

/* Device pointers of a problem (GraphSlice members, csr_problem.cuh:99-173). */
typedef struct b40c_bfs_device_view {
    void *d_row_offsets;    /* int32[nodes + 1] */
    void *d_column_indices; /* int32[edges] */
    void *d_labels;         /* int32[nodes] */
    void *d_visited_mask;   /* bit v&7 of byte v>>3 (same layout as the reference's uchar mask);
                               vertices without edges also have their bit set */
    int64_t visited_mask_bytes;
    int64_t nodes;
    int64_t edges;
    int32_t device;
    int32_t mark_predecessors;
} b40c_bfs_device_view;

/* ---- library ---------------------------------------------------------------- */

/* Text of the last error raised on the calling thread ("" if none). */
const char *b40c_last_error_string(void);

/* Library version string. */
const char *b40c_version(void);

/* Number of CUDA devices visible (0 on a machine without a GPU). */
int b40c_device_count(int *count);

/* Fills *policy with the tuned default for a strategy. */
int b40c_bfs_default_policy(int strategy, b40c_bfs_policy *policy);

/* ---- problem (bfs::CsrProblem, csr_problem.cuh:72-756) ---------------------- */

/* CsrProblem::FromHostProblem (csr_problem.cuh:328-540): copies the CSR to the
 * device (or, with stream_from_host, maps the caller's host arrays zero-copy,
 * pinning them in place when they are not page-locked yet: they must stay
 * valid until destroy; the kernels then read them over the bus with plain
 * loads).  Both arrays must be 4-byte aligned (B40C_ERROR_INVALID_VALUE
 * otherwise); no stronger alignment is needed.  device < 0 selects the
 * calling thread's current CUDA device.  num_gpus other than 1 is
 * rejected by the C++ layer (single-GPU library). */
int b40c_bfs_problem_create(const int32_t *h_row_offsets, const int32_t *h_column_indices,
                            int64_t nodes, int64_t edges, int mark_predecessors,
                            int stream_from_host, int device, b40c_bfs_problem **out);

/* CsrProblem::~CsrProblem (csr_problem.cuh:205-215). */
int b40c_bfs_problem_destroy(b40c_bfs_problem *problem);

/* Orders the handle's work on a caller stream (a cudaStream_t); NULL restores
 * the handle's own stream. */
int b40c_bfs_set_stream(b40c_bfs_problem *problem, void *cuda_stream);

/* Device bytes the handle holds now (CSR copy, labels, masks, queues, batch
 * buffers).  No counterpart in the reference (its GraphSlice allocations are
 * not reported, csr_problem.cuh:96-172). */
int b40c_bfs_problem_device_bytes(b40c_bfs_problem *problem, int64_t *bytes);

/* CsrProblem::Reset (csr_problem.cuh:547-750): (re)allocates the frontier
 * queues for frontier_type at queue_sizing x n (vertex) or x m (edge)
 * elements, and initialises labels to -1 and the visited mask to 0. */
int b40c_bfs_problem_reset(b40c_bfs_problem *problem, int frontier_type, double queue_sizing);

/* Enact{Fused,Iterative}Search / EnactSearch (enactor_contract_expand.cuh:262,419;
 * enactor_expand_contract.cuh; enactor_two_phase.cuh:276,421;
 * enactor_hybrid.cuh:279).  Searches from src; labels become source
 * distances (src = 0), or predecessors (src = -2) when the problem marks
 * predecessors; unreached vertices keep -1.  max_grid_size 0 = SMs x
 * occupancy (EnactorBase::MaxGridSize, enactor_base.cuh:93).  policy NULL =
 * tuned default.  Asynchronous apart from the iterative mode's per-level
 * frontier reads; b40c_bfs_stats or b40c_bfs_extract synchronise. */
int b40c_bfs_enact(b40c_bfs_problem *problem, int strategy, int mode, int32_t src,
                   int max_grid_size, const b40c_bfs_policy *policy);

/* Same as b40c_bfs_enact with a depth limit: vertices farther than
 * depth_limit levels from src stay -1 (depth_limit < 0: unlimited). */
int b40c_bfs_enact_limited(b40c_bfs_problem *problem, int strategy, int mode, int32_t src,
                           int32_t depth_limit, int max_grid_size, const b40c_bfs_policy *policy);

/* CsrProblem::ExtractResults (csr_problem.cuh:255-322): copies labels[n] to the host. */
int b40c_bfs_extract(b40c_bfs_problem *problem, int32_t *h_labels);

/* ExtractResults for pipelined searches (no reference counterpart: the
 * reference reads results back synchronously).  Copies the labels of the
 * search last enacted into device staging slot `slot` (0 or 1) in stream
 * order, then starts their device-to-host copy into h_labels (labels[n]; pinned
 * host memory lets it overlap) on a copy stream of the problem, and returns at
 * once: the next search may be enacted right away, it waits only for the
 * device-side copy.  A slot still in flight is waited for first.
 * b40c_bfs_extract_wait(slot) blocks until that slot's labels are in host
 * memory and returns the search's status (as b40c_bfs_extract would); it
 * returns at once for a slot with nothing in flight.  h_labels must stay valid
 * and untouched until then. */
int b40c_bfs_extract_async(b40c_bfs_problem *problem, int32_t *h_labels, int slot);
int b40c_bfs_extract_wait(b40c_bfs_problem *problem, int slot);

/* Enactor*::GetStatistics (enactor_contract_expand.cuh:237-250 and peers):
 * total_queued = sum of the frontier-queue lengths the search processed,
 * search_depth = number of BFS levels (max distance + 1), avg_duty = mean
 * fraction of each CTA's lifetime spent on work (0 unless instrumented). */
int b40c_bfs_stats(b40c_bfs_problem *problem, int64_t *total_queued, int32_t *search_depth,
                   double *avg_duty);

/* Whether the CSR is symmetric (every edge u->v has a matching v->u, as a
 * multiset), tested on the device by comparing order-independent 64-bit
 * hash sums of the edges and of their reversals; cached per problem.
 * Direction-optimizing searches run bottom-up levels only on symmetric graphs. */
int b40c_bfs_problem_is_symmetric(b40c_bfs_problem *problem, int *symmetric);

/* Instrumentation (the reference's INSTRUMENT template flag,
 * kernel_runtime_stats.cuh:45-126, and its driver's per-level histogram,
 * test_bfs.cu:264-337).  When on, each search records one entry per pass
 * (a level; edge strategies: contract and expand phases of a level) and the
 * CTAs' busy time, which b40c_bfs_stats reports as avg_duty. */
typedef struct b40c_level_record {
    int32_t vertices;  /* frontier entries (or edge-frontier items) processed by the pass */
    int32_t edges;     /* edges of the vertex frontier (0 for edge-frontier passes) */
    int32_t bottom_up; /* 1 when the level ran bottom-up */
    int32_t pass;      /* pass index; -1 marks the closing record */
    uint64_t t_ns;     /* device global timer when the pass started (closing record: search end) */
} b40c_level_record;

int b40c_bfs_set_instrument(b40c_bfs_problem *problem, int on);

/* Per-CTA times (%globaltimer ns) of the last instrumented persistent search,
 * out[(pass * ctas + cta) * 8 + phase] for the first max_passes (<= 64)
 * passes; phase 7 is the CTA's arrival at the end-of-level grid barrier,
 * phases 0-5 steps of its first work chunk of a top-down level (start,
 * frontier entries loaded, gather set up, gathered, discovered, emitted); 0
 * where a CTA did not get there.  The spread of a pass's arrivals is its load
 * imbalance (the per-CTA clocks of the reference's KernelRuntimeStats,
 * util/kernel_runtime_stats.cuh:45-126).  out needs max_passes x 2048 x 8 entries. */
int b40c_bfs_cta_arrivals(b40c_bfs_problem *problem, uint64_t *out, int max_passes, int *ctas);

/* Copies the last instrumented search's records (at most max_records) plus a
 * closing record; *count receives the number written. */
int b40c_bfs_level_records(b40c_bfs_problem *problem, b40c_level_record *out, int max_records, int *count);

/* Device time of the last enact in milliseconds (CUDA events on the handle's stream). */
int b40c_bfs_last_elapsed_ms(b40c_bfs_problem *problem, float *ms);

/* Device times (ms) of the search kernels of the last `count` enacts (oldest
 * first; at most 256 are kept): each spans from after the source set-up to
 * the end of the last level, per launch mode.  Synchronises on the newest. */
int b40c_bfs_recent_search_ms(b40c_bfs_problem *problem, int count, float *out);

/* GraphSlice device pointers (csr_problem.cuh:99-173). */
int b40c_bfs_device_view_get(b40c_bfs_problem *problem, b40c_bfs_device_view *view);

/* ---- batched multi-source search (no counterpart in the reference) ----------
 * Up to 64 sources searched together: one pass over each level's adjacency
 * lists serves every source (64-bit per-vertex visited / frontier masks;
 * dense levels of a symmetric graph pull instead of push).  The labels of
 * slot s are what a single-source search from sources[s] with
 * depth_limits[s] produces (distances; -1 unreached or beyond the limit).
 * depth_limits may be NULL (unlimited).  Duplicate sources are allowed.  One
 * persistent cooperative grid, asynchronous like b40c_bfs_enact (the
 * sources travel as kernel arguments, so batches may be queued back to back);
 * b40c_bfs_stats reports the deepest search as search_depth and
 * b40c_msbfs_stats each slot's own. */
int b40c_msbfs_enact(b40c_bfs_problem *problem, const int32_t *sources, const int32_t *depth_limits, int k,
                     int max_grid_size, const b40c_bfs_policy *policy);

/* Adds a source to the batch in flight (no counterpart in the reference):
 * the running search takes the request at its next level boundary and from
 * then on searches from `source` in slot `slot` too, alongside the batch's
 * sources; that slot's labels (and search depth) are those of a search from
 * `source` alone with `depth_limit`.  slot must lie in [k, rows), k the
 * batch's sources and rows the label rows the problem holds (the widest batch
 * it has run; at most 64); at most 64 requests per batch.  Asynchronous and
 * cheap (three small host-to-device copies on a stream of the problem's own):
 * it may be called while the batch runs.  A request that arrives after the
 * search ended is not taken: b40c_msbfs_joined reports how many were. */
int b40c_msbfs_join(b40c_bfs_problem *problem, int32_t slot, int32_t source, int32_t depth_limit);

/* After a batch: *taken = the number of b40c_msbfs_join requests the search
 * took (the first *taken, in call order); search_depths (NULL or [64]) gets
 * every slot's search depth. */
int b40c_msbfs_joined(b40c_bfs_problem *problem, int32_t *taken, int32_t *search_depths);

/* Copies slot `slot`'s labels of the last batch to the host (slots past k:
 * the sources that joined it). */
int b40c_msbfs_extract(b40c_bfs_problem *problem, int slot, int32_t *h_labels);

/* search_depths[k]: each slot's search depth in the last batch (max label + 1,
 * the GetStatistics meaning, enactor_contract_expand.cuh:237-250). */
int b40c_msbfs_stats(b40c_bfs_problem *problem, int32_t *search_depths);

/* Device array int32[k][nodes] of the last batch's labels (valid until the next batch). */
int b40c_msbfs_device_labels(b40c_bfs_problem *problem, void **d_labels, int32_t *k);

/* ---- search without allocation ----------------------------------------------
 * No counterpart in the reference.  A single-source distance search for
 * callers that cannot allocate device memory when they search -- code living
 * inside another allocator's pool or a fixed memory budget, a device whose
 * memory is already spoken for, or a latency-critical path where cudaMalloc /
 * cudaFree would stall.  The caller passes the CSR (d_row_offsets[nodes + 1],
 * d_column_indices[edges]) and the output d_labels[nodes], all device
 * pointers it owns; the visited mask, frontier queues and search state live
 * in a fixed scratch array built into the library (about 6.3 MB held on every
 * device that loads it, until the process exits).  Limits: at most 262,144
 * vertices and 4,194,304 edges; larger graphs are rejected with
 * B40C_ERROR_INVALID_VALUE (use b40c_bfs_problem_create).  The three arrays
 * must be 4-byte aligned (else B40C_ERROR_INVALID_VALUE); the column array
 * need not be 16-byte aligned (bulk copies of it are aligned by address).
 * The first call on a device sets that device up (looks up the scratch's
 * device address and the kernel's launch shape), so make it before any
 * stream capture, and do not call it after a cudaDeviceReset in the same
 * process (the set-up belongs to the context that was reset).  Every
 * call shares the one scratch array: calls whose work overlaps on the GPU
 * (different streams or threads at once) race and must be serialised by the
 * caller.  Runs on cuda_stream (NULL: the legacy default stream) on the
 * current device and returns when the search has finished; labels are the
 * same as b40c_bfs_enact's expand-contract distances. */
int b40c_bfs_search_noalloc(const int32_t *d_row_offsets, const int32_t *d_column_indices, int64_t nodes,
                            int64_t edges, int32_t src, int32_t *d_labels, void *cuda_stream);

/* ---- pinned host memory (CsrGraph(pinned), csr_graph.cuh:81-93) ------------ */
int b40c_host_alloc(void **ptr, size_t bytes, int mapped);
int b40c_host_free(void *ptr);

/* ---- graph builders (the b40c/graph/builder headers) ---------------------------
 * Native, multi-threaded builders used by the benchmark and the Python layer.
 * Arrays are allocated with malloc (or pinned when pinned != 0) and released
 * with b40c_graph_free.  Results are deterministic for a seed, independent of
 * the thread count. */
typedef struct b40c_csr {
    int64_t nodes;
    int64_t edges;
    int32_t *row_offsets;    /* [nodes + 1] */
    int32_t *column_indices; /* [edges] */
    int32_t pinned;
} b40c_csr;

/* BuildGrid2dGraph (grid2d.cuh:54-114): width^2 vertices, neighbour order
 * -x,+x,-y,+y, then a self-loop. */
int b40c_build_grid2d(int32_t width, int pinned, b40c_csr *out);

/* BuildGrid3dGraph (grid3d.cuh:54-129): width^3 vertices, neighbour order
 * -x,+x,-y,+y,-z,+z, then a self-loop. */
int b40c_build_grid3d(int32_t width, int pinned, b40c_csr *out);

/* COO -> CSR on the GPU (CsrGraph::FromCoo, csr_graph.cuh:109-152, done on
 * the device): d_rows/d_cols[edges] device arrays of 0-based ids are turned
 * into d_row_offsets[nodes + 1] and d_column_indices[edges] with rows in
 * input order (a stable radix sort by row).  Ids outside [0, nodes) return
 * B40C_ERROR_INVALID_VALUE.  Synchronous on cuda_stream; temporary device
 * memory of about 16 bytes per edge is allocated and freed inside. */
int b40c_coo_to_csr_device(const int32_t *d_rows, const int32_t *d_cols, int64_t nodes, int64_t edges,
                           int32_t *d_row_offsets, int32_t *d_column_indices, void *cuda_stream);

/* A problem handle built from a host COO edge list (FromCoo + FromHostProblem
 * in one step): the list is uploaded and converted on the GPU. */
int b40c_bfs_problem_create_coo(const int32_t *h_rows, const int32_t *h_cols, int64_t nodes, int64_t edges,
                                int mark_predecessors, int device, b40c_bfs_problem **out);

/* Graph files (path NULL = standard input).  Return 0, or
 * B40C_ERROR_INVALID_VALUE with the parse error in b40c_last_error_string().
 * Vertex ids in the files are 1-based; rows keep file order (FromCoo's
 * stable by-row sort, csr_graph.cuh:109-152).
 *   b40c_read_market  -- ReadMarketStream (market.cuh:49-160): "rows cols nnz",
 *                        then "col row [value]" lines; `undirected` adds each
 *                        entry's reverse edge right after it.
 *   b40c_read_dimacs  -- ReadDimacsStream (dimacs.cuh:52-228): "p <type> n m",
 *                        "a u v [w]" arcs; `splice` > 0 merges <path>.0,
 *                        <path>.1, ... by smallest row; `undirected` adds each
 *                        arc's reverse edge ahead of it.
 *   b40c_read_metis   -- ReadMetisStream (metis.cuh:51-187): "n m", then one
 *                        adjacency line per vertex; 2m (or m) ids expected. */
int b40c_read_market(const char *path, int undirected, int pinned, b40c_csr *out);
int b40c_read_dimacs(const char *path, int undirected, int splice, int pinned, b40c_csr *out);
int b40c_read_metis(const char *path, int pinned, b40c_csr *out);

/* BuildRmatGraph (rmat.cuh:128-206): `edges` R-MAT draws over `nodes` (a power
 * of two) with per-level +-5% parameter noise (VaryParams, rmat.cuh:83-116),
 * walk starting at u = v = 1 (rmat.cuh:167-169; the id `nodes` wraps to 0),
 * back-edges when undirected, self-loops and duplicates kept, rows in
 * generation order (FromCoo's stable sort, csr_graph.cuh:109-152).  With
 * permute != 0 vertex ids are relabelled by a seeded random permutation. */
int b40c_build_rmat(int64_t nodes, int64_t edges, int undirected, double a, double b, double c,
                    uint64_t seed, int permute, int pinned, b40c_csr *out);

/* BuildRandomGraph (random.cuh:54-98): `edges` uniform (u, v) pairs, back-edges when undirected. */
int b40c_build_random(int64_t nodes, int64_t edges, int undirected, uint64_t seed, int pinned,
                      b40c_csr *out);

/* BuildRandomRegularishGraph (rr.cuh:53-91): `degree` uniform out-neighbours
 * per vertex; with symmetrize != 0 every edge also gets its back-edge (the
 * random.cuh:81-86 construction) and rows keep generation order. */
int b40c_build_rr(int64_t nodes, int32_t degree, int symmetrize, uint64_t seed, int pinned,
                  b40c_csr *out);

/* CsrGraph::FromCoo (csr_graph.cuh:109-152): stable by-row CSR of a COO list. */
int b40c_csr_from_coo(const int32_t *rows, const int32_t *cols, int64_t nodes, int64_t edges,
                      int pinned, b40c_csr *out);

/* Seeded sample of `count` distinct vertices with nonzero degree (sources). */
int b40c_sample_sources(const b40c_csr *graph, int32_t count, uint64_t seed, int32_t *out);

void b40c_graph_free(b40c_csr *graph);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* B40C_BFS_H */
