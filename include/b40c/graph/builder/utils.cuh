/*
 * Builder helpers (drop-in for b40c/graph/builder/utils.cuh:55-61 and the
 * libc-rand() bit source of b40c/util/random_bits.cuh:62-88).
 *
 * The random builders of this header set draw from libc rand() in the same
 * order as the reference builders, so after the same srand() seed they build
 * the same graphs (on the same libc).  For large seeded graphs independent of
 * libc use the library's parallel builders (b40c_build_* in b40c_bfs.h).
 */
#pragma once
#include <stdlib.h>
#include <string.h>

#include "../csr_graph.cuh"

namespace b40c {
namespace graph {
namespace builder {

/* A key of random bits: one rand() call per byte, bits 7..14 of each draw. */
template <typename K>
void RandomBits(K &key)
{
    unsigned char bytes[sizeof(K)];
    for (size_t j = 0; j < sizeof(K); j++) bytes[j] = (unsigned char)(0xff & (rand() >> 7));
    memcpy(&key, bytes, sizeof(K));
}

/* A random vertex id in [0, num_nodes). */
template <typename SizeT>
SizeT RandomNode(SizeT num_nodes)
{
    SizeT node_id;
    RandomBits(node_id);
    long long x = (long long)node_id;
    if (x < 0) x = -x;
    return (SizeT)(x % (long long)num_nodes);
}

}  // namespace builder
}  // namespace graph
}  // namespace b40c
