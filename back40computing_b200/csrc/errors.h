// Thread-local error text for the C ABI (the reference prints every failure
// through B40CPerror, error_utils.cuh:44-108, and returns the cudaError_t;
// here the text is kept for b40c_last_error_string() and optionally echoed to
// stderr when B40C_VERBOSE_ERRORS is set).
#pragma once
#include <cstdarg>
#include <cstdio>
#include <cstdlib>

namespace b40c {

inline char *error_buffer()
{
    static thread_local char buf[512] = {0};
    return buf;
}

inline void clear_error() { error_buffer()[0] = 0; }

inline int fail(int code, const char *fmt, ...)
{
    char *buf = error_buffer();
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, 512, fmt, ap);
    va_end(ap);
    if (getenv("B40C_VERBOSE_ERRORS")) fprintf(stderr, "b40c: %s (status %d)\n", buf, code);
    return code;
}

}  // namespace b40c
