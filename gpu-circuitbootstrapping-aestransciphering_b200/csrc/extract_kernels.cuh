// extract_kernels.cuh -- launch interfaces of extract_kernels.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace cbs {

struct ExtractArgs {
    const uint64_t* words;  // [words][2][N] coefficient domain
    const uint32_t* info;   // [count] (word << 16) | coefficient
    const uint16_t* ksk;    // [2][N][base_ks][ksk_stride] (rows of n + 1 words padded to a multiple of 4)
    uint32_t ksk_stride;
    uint64_t* out_a;        // [count][out_stride]
    uint64_t* out_b;        // [count]
    uint32_t out_stride;
    uint32_t N, n;
    uint64_t Q;
    double q_over_Q;        // qks / Q
    uint32_t qks, mask;     // qks - 1
    uint32_t base_ks, base_log2;
    uint64_t q_lwe;
    uint64_t scale;         // q_lwe / qks when divisible, else 0
};

cudaError_t launch_extract_keyswitch(const ExtractArgs& a, uint32_t count, cudaStream_t s);
// row stride of the device key-switching key: n + 1 rounded up to a multiple of 4 words
inline uint32_t ksk_row_stride(uint32_t n) { return (n + 1 + 3) & ~3u; }
cudaError_t launch_init_state(uint64_t* out_a, uint64_t* out_b, const uint64_t* rk_a, const uint64_t* rk_b,
                              const uint8_t* bits, uint64_t half, uint64_t q, uint32_t n, uint32_t total,
                              cudaStream_t s);
// b[t] += q/2 (mod q) where bit t of bytes is set (bit t = byte t/8, bit t%8)
cudaError_t launch_add_public_bits(uint64_t* b, const uint8_t* bytes, uint64_t half, uint64_t q, uint32_t total,
                                   cudaStream_t s);
cudaError_t launch_assemble_words(uint64_t* words, const uint64_t* lut_out, const uint64_t* rk, uint64_t Q, uint32_t N,
                                  uint32_t blocks, cudaStream_t s);

}  // namespace cbs
