// Stand-in for the reference's umbrella header "phantom.h" when its example header
// bitwise/examples/aes_gpu_ks.cuh is compiled alone (ref_gpu_extract_shim.cu): only the CUDA
// runtime and the two error-check macros that header uses.  Test infrastructure.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#define PHANTOM_CHECK_CUDA(call)                                                          \
    do {                                                                                  \
        const cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string(cudaGetErrorString(e_))); \
    } while (0)
#define PHANTOM_CHECK_CUDA_LAST() PHANTOM_CHECK_CUDA(cudaGetLastError())
