/*
 * The data-model macro of b40c/util/cuda_properties.cuh:116-124 that callers
 * of the multi-GPU enactor test (test/bfs/test_bfs.cu checks it before
 * running on several GPUs): 1 when host pointers are 64-bit.
 */
#pragma once

#ifndef __B40C_LP64__
#if defined(_WIN64) || defined(__LP64__)
#define __B40C_LP64__ 1
#else
#define __B40C_LP64__ 0
#endif
#endif
