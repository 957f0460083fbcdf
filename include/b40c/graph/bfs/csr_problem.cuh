/*
 * BFS problem (drop-in for b40c/graph/bfs/csr_problem.cuh:54-756): device
 * copy of the CSR plus per-search labels, visited mask and frontier queues,
 * all owned by a libb40c_bfs problem handle.
 *
 * FromHostProblem / Reset / ExtractResults keep the reference's signatures and
 * cudaError_t results.  graph_slices[0] exposes the device arrays
 * (d_row_offsets, d_column_indices, d_labels, d_visited_mask: bit v & 7 of
 * byte v >> 3, as in the reference).  Only num_gpus == 1 is supported.
 *
 * The device arrays hold 32-bit ids and offsets (SizeT must be 32-bit).  A
 * 64-bit VertexId (the reference driver's "g500" graphs, test_bfs.cu:1066-1090)
 * is accepted on the host: FromHostProblem narrows the column indices into
 * an int32 copy the problem keeps (the one mapped zero-copy with
 * stream_from_host), ExtractResults widens the labels back, and
 * graph_slices[0]->d_column_indices / d_labels are then NULL (the device
 * copies are int32: b40c_bfs_device_view_get gives them).
 */
#pragma once
#include <stdio.h>

#include <vector>

#include "../../util/error_utils.cuh"
#include "b40c_bfs.h"
#include "problem_type.cuh"

namespace b40c {
namespace graph {
namespace bfs {

enum FrontierType {
    VERTEX_FRONTIERS = B40C_VERTEX_FRONTIERS,
    EDGE_FRONTIERS = B40C_EDGE_FRONTIERS,
    MIXED_FRONTIERS = B40C_MIXED_FRONTIERS,
    MULTI_GPU_FRONTIERS = B40C_MULTI_GPU_FRONTIERS,
    MULTI_GPU_VERTEX_FRONTIER_SCALE = 2,
};

template <typename _VertexId, typename _SizeT, bool MARK_PREDECESSORS>
struct CsrProblem {
    typedef bfs::ProblemType<_VertexId, _SizeT, unsigned char, unsigned char, MARK_PREDECESSORS> ProblemType;
    typedef _VertexId VertexId;
    typedef _SizeT SizeT;
    typedef unsigned char VisitedMask;
    typedef unsigned char ValidFlag;

    // the library's device arrays are 32-bit (ids of a 64-bit VertexId are narrowed on the host)
    typedef char vertex_id_must_be_32_or_64_bit[sizeof(VertexId) == 4 || sizeof(VertexId) == 8 ? 1 : -1];
    typedef char size_t_must_be_32_bit[sizeof(SizeT) == 4 ? 1 : -1];
    enum { NARROW_IDS = sizeof(VertexId) != 4 };

    /* Per-GPU device state (csr_problem.cuh:99-173); one slice on one GPU here. */
    struct GraphSlice {
        int gpu;
        VertexId *d_column_indices;
        SizeT *d_row_offsets;
        VertexId *d_labels;
        VisitedMask *d_visited_mask;
        VertexId nodes;
        SizeT edges;
        cudaStream_t stream;

        GraphSlice(int gpu) : gpu(gpu), d_column_indices(NULL), d_row_offsets(NULL), d_labels(NULL),
                              d_visited_mask(NULL), nodes(0), edges(0), stream(0) {}
    };

    int num_gpus;
    SizeT nodes;
    SizeT edges;
    std::vector<GraphSlice *> graph_slices;
    b40c_bfs_problem *handle;  // the library problem
    std::vector<int32_t> narrow_ids;  // 64-bit VertexId: the int32 column indices (outlive the handle)

    CsrProblem() : num_gpus(0), nodes(0), edges(0), handle(NULL) {}

    virtual ~CsrProblem()
    {
        for (size_t i = 0; i < graph_slices.size(); i++) delete graph_slices[i];
        if (handle) b40c_bfs_problem_destroy(handle);
    }

    /* Copies the CSR to the current device (or, with stream_from_host, maps the
     * host arrays zero-copy; they must outlive the problem). */
    cudaError_t FromHostProblem(bool stream_from_host, SizeT nodes, SizeT edges, VertexId *h_column_indices,
                                SizeT *h_row_offsets, int num_gpus)
    {
        if (num_gpus != 1)
            return util::B40CPerror(cudaErrorInvalidValue, "CsrProblem: this library searches on one GPU", __FILE__,
                                    __LINE__);
        if (handle) b40c_bfs_problem_destroy(handle);
        handle = NULL;
        const int32_t *ids = (const int32_t *)h_column_indices;
        if (NARROW_IDS) {
            narrow_ids.resize(edges > 0 ? (size_t)edges : 1);
            for (SizeT e = 0; e < edges; e++) {
                const long long u = (long long)h_column_indices[e];
                if (u < 0 || u >= (long long)nodes)
                    return util::B40CPerror(cudaErrorInvalidValue, "CsrProblem: column index out of range", __FILE__,
                                            __LINE__);
                narrow_ids[e] = (int32_t)u;
            }
            ids = narrow_ids.data();
        }
        int rc = b40c_bfs_problem_create((const int32_t *)h_row_offsets, ids, nodes, edges, MARK_PREDECESSORS ? 1 : 0,
                                         stream_from_host ? 1 : 0, -1 /* the caller's current device */, &handle);
        if (rc) return util::B40CPerror(util::AsCudaError(rc), "CsrProblem FromHostProblem failed", __FILE__, __LINE__);
        this->nodes = nodes;
        this->edges = edges;
        this->num_gpus = 1;
        for (size_t i = 0; i < graph_slices.size(); i++) delete graph_slices[i];
        graph_slices.clear();
        b40c_bfs_device_view view;
        b40c_bfs_device_view_get(handle, &view);
        GraphSlice *slice = new GraphSlice(view.device);
        slice->d_row_offsets = (SizeT *)view.d_row_offsets;
        slice->d_column_indices = NARROW_IDS ? NULL : (VertexId *)view.d_column_indices;
        slice->d_labels = NARROW_IDS ? NULL : (VertexId *)view.d_labels;
        slice->d_visited_mask = (VisitedMask *)view.d_visited_mask;
        slice->nodes = nodes;
        slice->edges = edges;
        graph_slices.push_back(slice);
        return cudaSuccess;
    }

    /* Sizes the frontier queues for frontier_type (queue_sizing x n or x m
     * elements) and resets labels to -1 and the visited mask to 0. */
    cudaError_t Reset(FrontierType frontier_type, double queue_sizing)
    {
        if (!handle) return util::B40CPerror(cudaErrorInvalidValue, "CsrProblem Reset before FromHostProblem", __FILE__, __LINE__);
        int rc = b40c_bfs_problem_reset(handle, (int)frontier_type, queue_sizing);
        return rc ? util::B40CPerror(util::AsCudaError(rc), "CsrProblem Reset failed", __FILE__, __LINE__) : cudaSuccess;
    }

    /* Copies the labels (distances, or predecessors) into h_label[nodes]. */
    cudaError_t ExtractResults(VertexId *h_label)
    {
        if (!handle) return cudaErrorInvalidValue;
        int rc;
        if (NARROW_IDS) {
            std::vector<int32_t> narrow(nodes > 0 ? (size_t)nodes : 1);
            rc = b40c_bfs_extract(handle, narrow.data());
            if (!rc)
                for (SizeT v = 0; v < nodes; v++) h_label[v] = (VertexId)narrow[v];  // -1 / -2 sign-extend
        } else {
            rc = b40c_bfs_extract(handle, (int32_t *)h_label);
        }
        return rc ? util::B40CPerror(util::AsCudaError(rc), "CsrProblem ExtractResults failed", __FILE__, __LINE__)
                  : cudaSuccess;
    }

  private:
    CsrProblem(const CsrProblem &);
    CsrProblem &operator=(const CsrProblem &);
};

}  // namespace bfs
}  // namespace graph
}  // namespace b40c
