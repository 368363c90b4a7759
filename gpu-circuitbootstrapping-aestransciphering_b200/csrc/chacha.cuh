// chacha.cuh -- the device samplers shared by the AES-material encryption (encrypt.cu) and the
// key generation (keygen_device.cu): the ChaCha20 block function (RFC 8439 s2.3) addressed by
// (counter, nonce), the uniform residue floor(x q / 2^128) of its words 0-3 and the
// discrete-Gaussian sample of its words 4-5 by cumulative table.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "encrypt.cuh"

namespace cbs {

__device__ __forceinline__ uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

#define CBS_CHACHA_QR(a, b, c, d)                                                                  \
    a += b; d = rotl32(d ^ a, 16);                                                                 \
    c += d; b = rotl32(b ^ c, 12);                                                                 \
    a += b; d = rotl32(d ^ a, 8);                                                                  \
    c += d; b = rotl32(b ^ c, 7);

// RFC 8439 s2.3: 20 rounds (10 column + diagonal double rounds), output = state + input
__device__ __forceinline__ void chacha20_block(const ChachaKey& k, uint32_t counter, uint32_t n0, uint32_t n1,
                                               uint32_t out[6]) {
    uint32_t x[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, k.w[0], k.w[1], k.w[2], k.w[3],
                      k.w[4],      k.w[5],      k.w[6],      k.w[7],      counter, n0,     n1,     0u};
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        CBS_CHACHA_QR(x[0], x[4], x[8], x[12])
        CBS_CHACHA_QR(x[1], x[5], x[9], x[13])
        CBS_CHACHA_QR(x[2], x[6], x[10], x[14])
        CBS_CHACHA_QR(x[3], x[7], x[11], x[15])
        CBS_CHACHA_QR(x[0], x[5], x[10], x[15])
        CBS_CHACHA_QR(x[1], x[6], x[11], x[12])
        CBS_CHACHA_QR(x[2], x[7], x[8], x[13])
        CBS_CHACHA_QR(x[3], x[4], x[9], x[14])
    }
    // only words 0..5 are consumed
    out[0] = x[0] + 0x61707865u;
    out[1] = x[1] + 0x3320646eu;
    out[2] = x[2] + 0x79622d32u;
    out[3] = x[3] + 0x6b206574u;
    out[4] = x[4] + k.w[0];
    out[5] = x[5] + k.w[1];
}
#undef CBS_CHACHA_QR

// floor(x * q / 2^128) for x = hi 2^64 + lo
__device__ __forceinline__ uint64_t uniform_mod(const uint32_t w[6], uint64_t q) {
    const uint64_t lo = w[0] | (static_cast<uint64_t>(w[1]) << 32);
    const uint64_t hi = w[2] | (static_cast<uint64_t>(w[3]) << 32);
    const uint64_t c = __umul64hi(lo, q);
    const uint64_t low = hi * q;
    const uint64_t sum = low + c;
    return __umul64hi(hi, q) + (sum < low ? 1u : 0u);
}

__device__ __forceinline__ int64_t cdt_sample(const uint32_t w[6], const uint64_t* T, uint32_t len) {
    const uint64_t u = w[4] | (static_cast<uint64_t>(w[5]) << 32);
    const uint64_t v = u & 0x7fffffffffffffffull;
    int64_t mag = 0;
    for (uint32_t k = 0; k < len; ++k) mag += v >= __ldg(T + k) ? 1 : 0;
    return (u >> 63) ? -mag : mag;
}

}  // namespace cbs
