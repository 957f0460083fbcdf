/*
 * Error reporting of the b40c host API (drop-in for b40c/util/error_utils.cuh:44-108):
 * B40CPerror prints a failing status with its origin to stderr and returns it.
 */
#pragma once
#include <cuda_runtime_api.h>
#include <stdio.h>

#include "b40c_bfs.h"

namespace b40c {
namespace util {

inline cudaError_t B40CPerror(cudaError_t error, const char *message, const char *filename, int line,
                              bool print = true)
{
    if (error && print) {
        const char *detail = b40c_last_error_string();
        fprintf(stderr, "[%s, %d] %s (CUDA error %d%s%s)\n", filename, line, message, (int)error,
                (detail && detail[0]) ? ": " : "", detail ? detail : "");
        fflush(stderr);
    }
    return error;
}

inline cudaError_t B40CPerror(cudaError_t error, const char *filename, int line, bool print = true)
{
    return B40CPerror(error, "b40c error", filename, line, print);
}

// Library status (int) as the cudaError_t the reference returns for it.
inline cudaError_t AsCudaError(int status) { return (cudaError_t)status; }

}  // namespace util
}  // namespace b40c
