// common.cuh -- status handling shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "../../include/cbs_b200.h"

namespace cbs {

void set_error(const std::string& msg);

// Status-returning CUDA check: records the failing call and returns CBS_ERR_CUDA.
#define CBS_CUDA_TRY(expr)                                                                     \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            ::cbs::set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));              \
            return (e_ == cudaErrorMemoryAllocation) ? CBS_ERR_OOM : CBS_ERR_CUDA;             \
        }                                                                                      \
    } while (0)

#define CBS_CHECK_ARG(cond, msg)                                                               \
    do {                                                                                       \
        if (!(cond)) {                                                                         \
            ::cbs::set_error(msg);                                                             \
            return CBS_ERR_INVALID_ARG;                                                        \
        }                                                                                      \
    } while (0)

#define CBS_LAUNCH_CHECK()                                                                     \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess) {                                                               \
            ::cbs::set_error(std::string("kernel launch: ") + cudaGetErrorString(e_));         \
            return CBS_ERR_CUDA;                                                               \
        }                                                                                      \
    } while (0)

inline int ilog2(uint64_t x) {
    int r = 0;
    while ((uint64_t(1) << r) < x) ++r;
    return r;
}

}  // namespace cbs
