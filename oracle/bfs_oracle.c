/*
 * CPU oracle for the single-source BFS path.  TEST INFRASTRUCTURE ONLY: the
 * product library never links, loads or calls anything in this directory;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * and only as the checker or the timed CPU baseline.
 *
 * Each function restates one piece of the reference driver test/bfs/test_bfs.cu
 * (b40c v1.0.1042) in plain C:
 *
 *   oracle_bfs                 SimpleReferenceBfs, test_bfs.cu:503-578
 *                              (FIFO order, labels -1 initialised, label = parent + 1,
 *                               search depth = max label + 1)
 *   oracle_bfs_limited         the same traversal stopped after a depth limit
 *                              (used to check depth-limited served queries)
 *   oracle_check_predecessors  the predecessor validity test, test_bfs.cu:387-439
 *   oracle_visited_stats       nodes/edges visited, test_bfs.cu:359-367
 *   oracle_compare_labels      CompareResults, test/b40c_test_util.h:304-336
 *
 * Parity of this restatement is pinned against the reference's own
 * SimpleReferenceBfs compiled from its source (oracle/build_ref.sh ->
 * oracle/_ref/libb40c_ref.so) and against the analytic lattice distances.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* test_bfs.cu:503-578.  Returns search_depth (max label + 1), or -1 on a bad
 * argument.  labels[n] receives source distances (-1 = unreached). */
int64_t oracle_bfs_limited(int64_t nodes, const int32_t *row_offsets,
                           const int32_t *column_indices, int32_t src,
                           int32_t depth_limit, int32_t *labels)
{
    if (nodes <= 0 || src < 0 || src >= nodes) return -1;
    for (int64_t i = 0; i < nodes; i++) labels[i] = -1;
    /* each vertex enters the FIFO at most once, so an n-slot array is the deque */
    int32_t *fifo = (int32_t *)malloc(sizeof(int32_t) * (size_t)nodes);
    if (!fifo) return -1;
    int64_t head = 0, tail = 0;
    int32_t search_depth = 0;
    labels[src] = 0;
    fifo[tail++] = src;
    while (head < tail) {
        int32_t u = fifo[head++];
        int32_t nd = labels[u] + 1;
        if (depth_limit >= 0 && nd > depth_limit) continue;
        for (int32_t e = row_offsets[u]; e < row_offsets[u + 1]; e++) {
            int32_t v = column_indices[e];
            if (labels[v] == -1) {
                labels[v] = nd;
                if (search_depth < nd) search_depth = nd;
                fifo[tail++] = v;
            }
        }
    }
    free(fifo);
    return (int64_t)search_depth + 1;
}

int64_t oracle_bfs(int64_t nodes, const int32_t *row_offsets,
                   const int32_t *column_indices, int32_t src, int32_t *labels)
{
    return oracle_bfs_limited(nodes, row_offsets, column_indices, src, -1, labels);
}

/* test_bfs.cu:387-439.  Returns -1 when every predecessor is plausible,
 * otherwise the first offending node.  *reason receives 1 (parentless node
 * with positive distance), 2 (parent not one level up) or 3 (parent is not
 * adjacent to the node). */
int64_t oracle_check_predecessors(int64_t nodes, const int32_t *row_offsets,
                                  const int32_t *column_indices,
                                  const int32_t *ref_dist, const int32_t *preds,
                                  int32_t *reason)
{
    *reason = 0;
    for (int64_t node = 0; node < nodes; node++) {
        int32_t parent = preds[node];
        if (parent < 0) {
            if (ref_dist[node] > 0) { *reason = 1; return node; }
            continue;
        }
        if (parent >= nodes) { *reason = 3; return node; }
        if (ref_dist[parent] + 1 != ref_dist[node]) { *reason = 2; return node; }
        int found = 0;
        for (int32_t e = row_offsets[parent]; e < row_offsets[parent + 1]; e++) {
            if (column_indices[e] == (int32_t)node) { found = 1; break; }
        }
        if (!found) { *reason = 3; return node; }
    }
    return -1;
}

/* test_bfs.cu:359-367: a vertex counts as visited when its label is > -1;
 * its full CSR row length (self-loops and duplicates included) counts as
 * visited edges. */
void oracle_visited_stats(int64_t nodes, const int32_t *row_offsets,
                          const int32_t *labels, int64_t *nodes_visited,
                          int64_t *edges_visited)
{
    int64_t nv = 0, ev = 0;
    for (int64_t i = 0; i < nodes; i++) {
        if (labels[i] > -1) {
            nv++;
            ev += row_offsets[i + 1] - row_offsets[i];
        }
    }
    *nodes_visited = nv;
    *edges_visited = ev;
}

/* b40c_test_util.h:304-336: returns -1 when equal, else the first mismatch. */
int64_t oracle_compare_labels(int64_t n, const int32_t *computed, const int32_t *reference)
{
    for (int64_t i = 0; i < n; i++)
        if (computed[i] != reference[i]) return i;
    return -1;
}

/* Per-level frontier sizes of a distance labelling: counts[d] = #{v : label[v] == d}
 * for d < max_levels.  Returns the number of levels (max label + 1). */
int64_t oracle_level_histogram(int64_t nodes, const int32_t *labels,
                               int64_t *counts, int64_t max_levels)
{
    int64_t levels = 0;
    for (int64_t d = 0; d < max_levels; d++) counts[d] = 0;
    for (int64_t i = 0; i < nodes; i++) {
        int32_t l = labels[i];
        if (l >= 0) {
            if (l < max_levels) counts[l]++;
            if (l + 1 > levels) levels = l + 1;
        }
    }
    return levels;
}
