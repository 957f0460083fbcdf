/*
 * b40c_server.h -- a BFS query server over several resident graphs.
 *
 * No counterpart in the reference, which runs one search at a time from its
 * test driver (test/bfs/test_bfs.cu:584-783, RunTests).  The server keeps
 * several CSR graphs resident on one GPU inside a fixed device-memory budget
 * and answers single-source BFS queries (source, optional depth limit) with
 * continuous batching: whenever the GPU can take more work, the queries that
 * have arrived for one graph (up to 64) are searched together by the batched
 * kernel (b40c_msbfs_enact); a lone query runs the plain single-source search
 * instead.  Every answer is what b40c_bfs_enact_limited / b40c_bfs_extract
 * would give for that query alone: labels are distances, -1 unreached or
 * beyond the depth limit, and search_depth is max label + 1.
 *
 * One background thread per server issues the GPU work (one CUDA stream per
 * in-flight slot) and retires finished batches; the calls below may come from
 * any thread.
 * A query that arrives while its graph's batched search is running joins
 * that search at its next level boundary when the batch has a free slot
 * (b40c_msbfs_join), instead of waiting for the next batch.
 * Status codes are the cudaError_t values of b40c_bfs.h.
 */
#ifndef B40C_SERVER_H
#define B40C_SERVER_H

#include <stdint.h>

#include "b40c_bfs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b40c_server b40c_server;

typedef struct b40c_server_options {
    /* Device bytes the server may hold for graphs and their search buffers
     * (CSR copy, labels, masks, frontier queues, batch buffers); 0 = 90% of
     * the device memory free when the server is created. */
    int64_t memory_budget_bytes;
    /* Most queries searched together, 1..64 (0 = 64).  A graph admitted when
     * the budget cannot hold its batch buffers at this width gets the widest
     * power-of-two width that fits. */
    int32_t max_batch;
    /* Strategy for a batch of one query: B40C_DIRECTION_OPTIMIZING (default,
     * 0 is read as this), B40C_EXPAND_CONTRACT, or -1 to use the batched
     * kernel for lone queries too. */
    int32_t single_strategy;
    /* Batches on the GPU at once, over all graphs (0 = 2); at most one per
     * graph, so queries for a busy graph gather into its next batch.  Each
     * in-flight batch has a CUDA stream of its own: batches of different
     * graphs, and one batch's label read-back with another's search, overlap. */
    int32_t max_in_flight;
    /* CTAs per SM of each batch's persistent grid: 0 = split the SMs evenly
     * among the max_in_flight slots (4 / max_in_flight, at least 1; the
     * kernels are resident at up to 4), so the grids of concurrent batches
     * are resident side by side; -1 = every batch takes the whole device
     * (concurrent batches then mostly wait for each other). */
    int32_t ctas_per_sm;
    int32_t reserved[4];
} b40c_server_options;

typedef struct b40c_server_result {
    int64_t ticket;
    int32_t graph, source, depth_limit;
    int32_t status;        /* 0, B40C_ERROR_NOT_READY (600) while pending, or the failure's code */
    int32_t search_depth;  /* max label + 1 */
    int32_t batch_size;    /* queries in the launch that answered it */
    int64_t arrival_ns;    /* server clock: when the query became eligible */
    int64_t launch_ns;     /* when its batch was issued to the GPU */
    int64_t finish_ns;     /* when the server saw its batch (and its label copy) finish */
    int64_t gpu_start_ns;  /* device clock (CUDA events on the batch's stream, from the server's creation):
                              when its batch's search began on the GPU ... */
    int64_t gpu_end_ns;    /* ... and when it ended (before the label copy) */
} b40c_server_result;

typedef struct b40c_server_counters {
    int64_t submitted, completed, failed;
    int64_t batches, batched_queries, single_queries;
    int64_t memory_used_bytes, memory_budget_bytes;
    int32_t graphs;
    int32_t reserved;
    int64_t joined_queries; /* of batched_queries: the ones that joined a batch in flight */
} b40c_server_counters;

/* options may be NULL (all defaults).  device < 0 = the current device. */
int b40c_server_create(int device, const b40c_server_options *options, b40c_server **out);

/* Waits for every submitted query, stops the thread and frees everything. */
int b40c_server_destroy(b40c_server *server);

/* Copies a host CSR graph to the device and admits it against the budget.
 * Returns B40C_ERROR_MEMORY_ALLOCATION (2) without changing anything when the
 * graph does not fit even at batch width 1.  *graph_id numbers graphs from 0. */
int b40c_server_add_graph(b40c_server *server, const int32_t *row_offsets, const int32_t *column_indices,
                          int64_t nodes, int64_t edges, int32_t *graph_id);

/* Frees a graph's memory; B40C_ERROR_NOT_READY (600) while it has queries
 * pending or in flight. */
int b40c_server_remove_graph(b40c_server *server, int32_t graph_id);

/* Kernel policies for a graph's lone-query searches and its batches (either
 * may be NULL: the library defaults); e.g. the autotuner's choice for the
 * graph's class.  Validated like b40c_bfs_enact's policy argument. */
int b40c_server_set_graph_policy(b40c_server *server, int32_t graph_id, const b40c_bfs_policy *single,
                                 const b40c_bfs_policy *batch);

/* Device bytes a graph holds and its batch width. */
int b40c_server_graph_info(b40c_server *server, int32_t graph_id, int64_t *device_bytes, int32_t *max_batch);

/* Device bytes a graph of this size would hold at batch width max_batch
 * (what admission charges against the budget). */
int b40c_server_plan_bytes(int64_t nodes, int64_t edges, int32_t max_batch, int64_t *device_bytes);

/* Server clock (steady, nanoseconds since the server was created). */
int b40c_server_now_ns(b40c_server *server, int64_t *now_ns);

/* Queues one query.  depth_limit < 0 = unlimited.  h_labels (may be NULL)
 * receives the query's labels (nodes int32 values) when it finishes.  Into
 * page-locked memory (b40c_host_alloc) the copy is queued behind the search
 * and overlaps other work; into pageable memory the server copies when the
 * search has finished (the dispatcher is busy for that copy only).  arrival_ns < 0 =
 * now; a future arrival time makes the query eligible only then (used to
 * replay a timed request stream).  *ticket identifies the query. */
int b40c_server_submit(b40c_server *server, int32_t graph_id, int32_t source, int32_t depth_limit,
                       int32_t *h_labels, int64_t arrival_ns, int64_t *ticket);

/* Queues count queries at once (labels not returned); tickets[] may be NULL.
 * Every query is checked before any is queued. */
int b40c_server_submit_many(b40c_server *server, int64_t count, const int32_t *graph_ids, const int32_t *sources,
                            const int32_t *depth_limits, const int64_t *arrival_ns, int64_t *tickets);

/* Result of one query; status B40C_ERROR_NOT_READY while it is pending. */
int b40c_server_result_get(b40c_server *server, int64_t ticket, b40c_server_result *out);

/* Blocks until the query has finished (its labels copied). */
int b40c_server_wait(b40c_server *server, int64_t ticket, b40c_server_result *out);

/* Blocks until every query submitted so far has finished. */
int b40c_server_drain(b40c_server *server);

/* Results of tickets [first, first + count). */
int b40c_server_results(b40c_server *server, int64_t first, int64_t count, b40c_server_result *out);

int b40c_server_counters_get(b40c_server *server, b40c_server_counters *out);

#ifdef __cplusplus
}
#endif

#endif /* B40C_SERVER_H */
