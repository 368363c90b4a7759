// noalloc.cu -- circuit bootstrapping for callers that cannot allocate device memory.
//
// cbs_circuit_bootstrap_batch_device() keeps its multi-value RLWEs (the hand-off between
// the blind rotation and the HomTrace kernels) in scratch that the context allocates with
// cudaMalloc.  Some callers cannot allocate at the time they bootstrap: code running inside
// a stream-capture region (a cudaMalloc there breaks or invalidates the capture), serving
// loops with latency budgets (cudaMalloc/cudaFree can synchronize the whole device), and
// components whose device memory is owned by another allocator that hands them no budget
// of their own.  This entry point serves them: the caller passes the inputs and the output
// buffer, and the intermediate lives in a fixed file-scope device array below.
#include <mutex>

#include "common.cuh"
#include "context.cuh"

namespace cbs {

// Capacity of the shared scratch in 64-bit words: 4 MiB, i.e. batch * num_lut * 2 * N words
// (32 ciphertexts at N = 2048 with 4 LUT levels).  Every GPU that loads this library keeps
// this array until the process exits.
static constexpr size_t kNoAllocScratchWords = size_t(1) << 19;

static __device__ __align__(256) uint64_t g_noalloc_scratch[kNoAllocScratchWords];

static constexpr int kMaxDevices = 64;
static uint64_t* g_scratch_addr[kMaxDevices] = {};
static std::mutex g_scratch_mu;

// The device address of g_noalloc_scratch on the current device.  The name of the array is
// only a host-side stand-in, so the address is queried once per device (with that device
// current) and cached.
static cbs_status scratch_address(uint64_t** out) {
    int dev = 0;
    CBS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("circuit_bootstrap_noalloc: device ordinal beyond the supported range");
        return CBS_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            set_error(std::string("circuit_bootstrap_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return CBS_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<uint64_t*>(p);
    }
    *out = g_scratch_addr[dev];
    return CBS_OK;
}

}  // namespace cbs

using namespace cbs;

extern "C" {

size_t cbs_circuit_bootstrap_noalloc_capacity_words(void) { return kNoAllocScratchWords; }

cbs_status cbs_circuit_bootstrap_batch_device_noalloc(cbs_context* ctx, const uint64_t* d_a, const uint64_t* d_b,
                                                      uint32_t batch, uint32_t a_stride, uint64_t* d_rgsw_out,
                                                      cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "circuit_bootstrap_noalloc: null context");
    if (batch == 0) return CBS_OK;
    CBS_CHECK_ARG(d_a && d_b && d_rgsw_out, "circuit_bootstrap_noalloc: null pointer");
    CBS_CHECK_ARG(a_stride >= ctx->p.n, "circuit_bootstrap_noalloc: a_stride < n");
    const size_t need = static_cast<size_t>(batch) * ctx->p.num_lut * 2 * ctx->p.N;
    if (need > kNoAllocScratchWords) {
        set_error("circuit_bootstrap_noalloc: batch * num_lut * 2 * N = " + std::to_string(need) +
                  " words exceeds the fixed scratch of " + std::to_string(kNoAllocScratchWords) +
                  " words; split the batch");
        return CBS_ERR_SHAPE_MISMATCH;
    }
    if (!ctx->keys_ready) {
        set_error("circuit_bootstrap_noalloc: no key material (call cbs_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    // the scratch address is per device: the current device must hold this context's keys
    int dev = -1;
    CBS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != ctx->device) {
        set_error("circuit_bootstrap_noalloc: the current device (" + std::to_string(dev) +
                  ") is not the context's device (" + std::to_string(ctx->device) +
                  "); call cudaSetDevice first");
        return CBS_ERR_INVALID_ARG;
    }
    uint64_t* scratch = nullptr;
    if (cbs_status st = scratch_address(&scratch)) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // the blind rotation writes every scratch word it hands to the trace kernel, so stale
    // contents from an earlier call need no clearing
    return run_cbs(ctx, d_a, d_b, batch, a_stride, scratch, d_rgsw_out, s);
}

}  // extern "C"
