// Status and error-message plumbing shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>

#include "ct2b200.h"

namespace ct2 {

// Records a formatted message for ct2_last_error() and returns `code`.
int set_error(int code, const char* fmt, ...);
// Clears the per-thread message; returns CT2_OK.
int clear_error();
// Counts one kernel launch of the library (ct2_launch_count).
void note_launch();

}  // namespace ct2

// Validation helper: bail out with CT2_EINVAL and a message.
#define CT2_REQUIRE(cond, ...)                                   \
    do {                                                         \
        if (!(cond)) return ct2::set_error(CT2_EINVAL, __VA_ARGS__); \
    } while (0)

// CUDA call helper: bail out with CT2_ECUDA and the CUDA error string.
#define CT2_CUDA(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ct2::set_error(e_ == cudaErrorMemoryAllocation ? CT2_ENOMEM : CT2_ECUDA, \
                                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),       \
                                  __FILE__, __LINE__);                                  \
    } while (0)

// After a kernel launch: count it, report a launch error.
#define CT2_LAUNCHED()            \
    do {                          \
        ct2::note_launch();       \
        CT2_CUDA(cudaGetLastError()); \
    } while (0)
