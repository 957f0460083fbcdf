/*
 * Small type utilities the graph headers use (the subset of
 * b40c/util/basic_utils.cuh the BFS host API needs).
 */
#pragma once
#include <stdio.h>

namespace b40c {
namespace util {

struct NullType {};

template <bool IF, typename ThenType, typename ElseType>
struct If {
    typedef ThenType Type;
};
template <typename ThenType, typename ElseType>
struct If<false, ThenType, ElseType> {
    typedef ElseType Type;
};

}  // namespace util

inline void PrintValue(int v) { printf("%d", v); }
inline void PrintValue(long long v) { printf("%lld", v); }
inline void PrintValue(unsigned int v) { printf("%u", v); }
inline void PrintValue(long v) { printf("%ld", v); }

}  // namespace b40c
