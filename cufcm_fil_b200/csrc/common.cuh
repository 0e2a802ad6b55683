// common.cuh -- status codes, thread-local error text and CUDA checks shared by
// every translation unit of libcufil.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdio>
#include <cstdarg>
#include <cstdlib>
#include <string>
#include <utility>

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

// Programmatic dependent launch for the kernels of the implicit step's inner loops
// (the GMRES iteration and the Gauss-Jordan rounds of the patch refresh).  A
// kernel launched by launch_chained() may be scheduled while the previous kernel
// of its stream drains (its blocks are scheduled as the previous kernel's blocks
// exit); it calls chain_wait() before it touches global memory, which returns
// once that kernel has completed and its writes are visible, so the stream's
// order is kept and only the launch latency between the kernels is hidden.
// chain_wait() is a no-op for an ordinary launch.  CUFIL_NO_PDL=1 makes
// launch_chained() an ordinary launch.
__device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

inline bool chained_launches() {
    static const bool on = [] {
        const char *v = std::getenv("CUFIL_NO_PDL");
        return !(v && *v && *v != '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                  Args &&...args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = chained_launches() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
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
