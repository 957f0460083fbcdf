/*
 * BFS problem type (drop-in for b40c/graph/bfs/problem_type.cuh:53-70).
 * The B200 library is single-GPU and uses 32-bit vertex ids and offsets; the
 * GPU-id bits keep their reference values for source compatibility.
 */
#pragma once
#include "../../util/basic_utils.cuh"

namespace b40c {
namespace graph {
namespace bfs {

template <typename _VertexId, typename _SizeT, typename _VisitedMask, typename _ValidFlag, bool _MARK_PREDECESSORS>
struct ProblemType {
    typedef _VertexId VertexId;
    typedef _SizeT SizeT;
    typedef _VisitedMask VisitedMask;
    typedef _ValidFlag ValidFlag;
    typedef typename util::If<_MARK_PREDECESSORS, _VertexId, util::NullType>::Type ValueType;

    static const bool MARK_PREDECESSORS = _MARK_PREDECESSORS;
    static const _VertexId LOG_MAX_GPUS = 2;
    static const _VertexId MAX_GPUS = 1 << LOG_MAX_GPUS;
    static const _VertexId GPU_MASK_SHIFT = (sizeof(_VertexId) * 8) - LOG_MAX_GPUS;
    static const _VertexId GPU_MASK = (MAX_GPUS - 1) << GPU_MASK_SHIFT;
    static const _VertexId VERTEX_ID_MASK = ~GPU_MASK;
};

}  // namespace bfs
}  // namespace graph
}  // namespace b40c
