// Expand-contract enactor and its kernel variants for 512-thread CTAs.
#include "enact_vertex_impl.cuh"

namespace b40c {
namespace rt {
template int enact_vertex_b<512>(b40c_bfs_problem *, int, int32_t, int, const b40c_bfs_policy &, int32_t, bool);
}  // namespace rt
}  // namespace b40c
