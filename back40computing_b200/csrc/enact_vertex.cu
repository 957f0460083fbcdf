// Expand-contract enactor (vertex frontiers): one persistent cooperative
// grid (fused), one launch per level (iterative), or a CUDA graph of the
// whole search with a conditional WHILE node over levels.  The body is in
// enact_vertex_impl.cuh, compiled once per CTA size (enact_vertex_<B>.cu).
#include "launch_common.cuh"

namespace b40c {
namespace rt {

template <int B>
int enact_vertex_b(b40c_bfs_problem *p, int mode, int32_t src, int max_grid, const b40c_bfs_policy &pol,
                   int32_t depth_limit, bool direction_optimizing);

int enact_vertex(b40c_bfs_problem *p, int mode, int32_t src, int max_grid, const b40c_bfs_policy &pol,
                 int32_t depth_limit, bool direction_optimizing)
{
    switch (pol.threads) {
    case 128: return enact_vertex_b<128>(p, mode, src, max_grid, pol, depth_limit, direction_optimizing);
    case 512: return enact_vertex_b<512>(p, mode, src, max_grid, pol, depth_limit, direction_optimizing);
    default: return enact_vertex_b<256>(p, mode, src, max_grid, pol, depth_limit, direction_optimizing);
    }
}

}  // namespace rt
}  // namespace b40c
