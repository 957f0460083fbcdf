// Edge-frontier strategies (contract-expand, two-phase, hybrid).
#pragma once
#include "b40c_bfs.h"
#include "errors.h"

namespace b40c {
inline int enact_edge_strategy(b40c_bfs_problem *, int strategy, int, int32_t, int, const b40c_bfs_policy &, int32_t)
{
    return b40c::fail(B40C_ERROR_NOT_SUPPORTED, "strategy %d not built yet", strategy);
}
}  // namespace b40c
