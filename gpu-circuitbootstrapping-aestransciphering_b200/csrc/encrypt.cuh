// encrypt.cuh -- device encryption of the AES material (encrypt.cu) and the host-built
// noise table it samples from.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/cbs_b200.h"

namespace cbs {

struct ChachaKey {
    uint32_t w[8];  // 256-bit key, little-endian words of the caller's 32 bytes
};

struct EncryptRlweArgs {
    ChachaKey key;
    const uint32_t* words;  // [count] plaintext words (bit j -> coefficient j); null = encryptions of 0
    uint64_t* ct;           // [count][2][N] out: (a, b), NTT domain
    uint64_t* tmp;          // [count][N] scratch
    const uint64_t* s_ntt;  // [N] NTT(s), normal form
    const uint64_t* cdt;    // cumulative noise table
    uint32_t cdt_len;
    uint32_t N;
    uint32_t first;         // sample index of words[0] (the ChaCha20 nonce)
    uint64_t Q, delta, ratio0, ratio1;
    uint32_t domain;        // second nonce word: 1 = AES material; key generation uses 4-9
};

struct EncryptLweArgs {
    ChachaKey key;
    const uint8_t* bits;  // [count] 0/1 messages (scaled by floor(q/2))
    const int32_t* s;     // [n] binary LWE secret
    const uint64_t* cdt;
    uint32_t cdt_len;
    uint32_t n, a_stride;
    uint64_t q;
    uint64_t* out_a;  // [count][a_stride]
    uint64_t* out_b;  // [count]
};

cudaError_t ntt_forward(uint64_t* out, const uint64_t* in, const uint64_t* tw, const uint64_t* tws,
                        const cbs_dmodulus* mod, size_t dim, size_t batch, cudaStream_t s);
// RLWE encryptions of count words (mask pass, forward NTT of e + m, b = a s + ...)
cudaError_t launch_encrypt_rlwe_words(const EncryptRlweArgs& a, uint32_t count, const uint64_t* rp,
                                      const uint64_t* rps, const cbs_dmodulus* mod, cudaStream_t s);
cudaError_t launch_encrypt_lwe_bits(const EncryptLweArgs& a, uint32_t count, cudaStream_t s);

// T[k] = floor(2^63 P(|X| <= k)) for the discrete Gaussian exp(-x^2 / 2 sigma^2), k = 0, 1, ...
// while below 2^63 (long double arithmetic)
std::vector<uint64_t> cdt_table(double sigma);

}  // namespace cbs
