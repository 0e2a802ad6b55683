// common.cuh -- status codes, thread-local error text and CUDA checks shared by
// every translation unit of libcufil.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdio>
#include <cstdarg>
#include <string>

#include "../../include/cufil.h"

namespace cufil {

// Records a message for cf_last_error() and returns the code unchanged.
int set_error(int code, const char *fmt, ...);
// Clears the thread-local message (called on entry by every C-ABI function).
void clear_error();

// Converts a CUDA error into CF_ECUDA with file/line context.
inline int cuda_status(cudaError_t e, const char *what, const char *file, int line) {
    if (e == cudaSuccess) return CF_OK;
    return set_error(e == cudaErrorMemoryAllocation ? CF_ENOMEM : CF_ECUDA, "%s failed at %s:%d: %s",
                     what, file, line, cudaGetErrorString(e));
}

}  // namespace cufil

#define CF_CUDA(call)                                                                 \
    do {                                                                              \
        cudaError_t cf_e_ = (call);                                                   \
        if (cf_e_ != cudaSuccess) return cufil::cuda_status(cf_e_, #call, __FILE__, __LINE__); \
    } while (0)

#define CF_CHECK_LAUNCH(name)                                                         \
    do {                                                                              \
        cudaError_t cf_e_ = cudaGetLastError();                                       \
        if (cf_e_ != cudaSuccess) return cufil::cuda_status(cf_e_, name, __FILE__, __LINE__); \
    } while (0)

#define CF_TRY(expr)                    \
    do {                                \
        int cf_rc_ = (expr);            \
        if (cf_rc_ != CF_OK) return cf_rc_; \
    } while (0)

#define CF_REQUIRE(cond, ...)                                   \
    do {                                                        \
        if (!(cond)) return cufil::set_error(CF_EINVAL, __VA_ARGS__); \
    } while (0)

// Number of SMs on a B200 (two dies x 74); launch shapes are sized against the
// value queried at handle creation, this is only the fallback.
#define CF_B200_SMS 148
