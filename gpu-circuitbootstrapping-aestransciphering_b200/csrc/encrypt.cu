// encrypt.cu -- encryption of the AES material on the device.
//
// The reference encrypts its 8 x 256 T-table words and round-key words as RLWE and the
// round-0 key bits as LWE on the host, one sample at a time (EncryptWord32RLWE /
// BuildTableRLWE, examples/aes_transcipher/rlwe_tables.cuh:5-24; BuildEncryptedKeyMaterial,
// key_material.cuh:12-46).  Here every coefficient of every sample is drawn independently:
//
//   randomness  ChaCha20 (RFC 8439 block function) in counter mode under the caller's
//               256-bit key, one 64-byte block per coefficient: block counter = coefficient
//               index, nonce = (sample index, domain, 0) with domain 1 for RLWE and 2 for
//               LWE samples.  The words do not depend on the launch shape, so the CPU
//               restatement reproduces each of them.
//   mask        words 0-3 as x < 2^128, coefficient floor(x * q / 2^128) (bias < q / 2^128);
//               RLWE masks are drawn in the NTT domain, like the host encryption.
//   noise       words 4-5 as u < 2^64: sign = bit 63, magnitude = #{k : (u mod 2^63) >= T[k]}
//               for the cumulative table T of the discrete Gaussian exp(-x^2 / 2 sigma^2)
//               (integer compares only; the table is built on the host).
//
// RLWE: b = a * s + NTT(e + m) with m = floor(Q/2) on coefficient j < 32 where bit j of the
// word is set; LWE: b = <a, s> + m + e mod q.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "arith.cuh"
#include "chacha.cuh"
#include "encrypt.cuh"

namespace cbs {

// pass 1 of the RLWE samples: masks (NTT domain) into ct[r][0], e + m (coefficient domain)
// into tmp[r]; one CTA per sample
__global__ void k_encrypt_rlwe_words(EncryptRlweArgs a) {
    const uint32_t r = blockIdx.x;
    const uint32_t w = a.words ? a.words[r] : 0u;
    const uint32_t N = a.N;
    uint64_t* ct = a.ct + static_cast<size_t>(r) * 2 * N;
    uint64_t* tmp = a.tmp + static_cast<size_t>(r) * N;
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
        uint32_t blk[6];
        chacha20_block(a.key, i, a.first + r, a.domain ? a.domain : 1u, blk);
        ct[i] = uniform_mod(blk, a.Q);
        const int64_t e = cdt_sample(blk, a.cdt, a.cdt_len);
        uint64_t v = e < 0 ? a.Q - static_cast<uint64_t>(-e) : static_cast<uint64_t>(e);
        if (i < 32 && ((w >> i) & 1u)) {
            v += a.delta;
            if (v >= a.Q) v -= a.Q;
        }
        tmp[i] = v;
    }
}

// pass 2 (after the forward NTT of tmp): b = a * s + tmp
__global__ void k_encrypt_rlwe_finish(EncryptRlweArgs a, uint32_t count) {
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<size_t>(count) * a.N) return;
    const uint32_t r = static_cast<uint32_t>(idx / a.N), i = static_cast<uint32_t>(idx % a.N);
    uint64_t* ct = a.ct + static_cast<size_t>(r) * 2 * a.N;
    uint64_t v = mul_mod_barrett(ct[i], a.s_ntt[i], a.Q, a.ratio0, a.ratio1) + a.tmp[idx];
    if (v >= a.Q) v -= a.Q;
    ct[a.N + i] = v;
}

// LWE samples of bits: one CTA per sample, block-reduced <a, s>
__global__ void k_encrypt_lwe_bits(EncryptLweArgs a) {
    __shared__ uint64_t part[32];
    const uint32_t t = blockIdx.x;
    uint64_t acc = 0;
    for (uint32_t i = threadIdx.x; i < a.n; i += blockDim.x) {
        uint32_t blk[6];
        chacha20_block(a.key, i, t, 2u, blk);
        const uint64_t ai = uniform_mod(blk, a.q);
        a.out_a[static_cast<size_t>(t) * a.a_stride + i] = ai;
        acc += a.s[i] ? ai : 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t sum = 0;
        for (uint32_t j = 0; j < (blockDim.x + 31) / 32; ++j) sum += part[j];
        uint32_t blk[6];
        chacha20_block(a.key, a.n, t, 2u, blk);
        const int64_t e = cdt_sample(blk, a.cdt, a.cdt_len);
        const uint64_t eq = e < 0 ? a.q - static_cast<uint64_t>(-e) % a.q : static_cast<uint64_t>(e) % a.q;
        const uint64_t m = a.bits[t] ? a.q >> 1 : 0;
        a.out_b[t] = (sum % a.q + m + eq) % a.q;
    }
}

cudaError_t launch_encrypt_rlwe_words(const EncryptRlweArgs& a, uint32_t count, const uint64_t* rp,
                                      const uint64_t* rps, const cbs_dmodulus* mod, cudaStream_t s) {
    if (!count) return cudaSuccess;
    k_encrypt_rlwe_words<<<count, 256, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = ntt_forward(a.tmp, a.tmp, rp, rps, mod, a.N, count, s);
    if (e != cudaSuccess) return e;
    const size_t work = static_cast<size_t>(count) * a.N;
    k_encrypt_rlwe_finish<<<static_cast<unsigned>((work + 255) / 256), 256, 0, s>>>(a, count);
    return cudaGetLastError();
}

cudaError_t launch_encrypt_lwe_bits(const EncryptLweArgs& a, uint32_t count, cudaStream_t s) {
    if (!count) return cudaSuccess;
    k_encrypt_lwe_bits<<<count, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace cbs

namespace cbs {

std::vector<uint64_t> cdt_table(double sigma) {
    std::vector<uint64_t> T;
    if (!(sigma > 0)) return T;  // no noise: every sample is 0
    const long double s2 = 2.0L * static_cast<long double>(sigma) * static_cast<long double>(sigma);
    const int X = static_cast<int>(std::ceil(14.0 * sigma)) + 1;
    long double S = 1.0L;
    for (int x = 1; x <= X; ++x) S += 2.0L * expl(-static_cast<long double>(x) * x / s2);
    const long double two63 = 9223372036854775808.0L;
    long double cum = 1.0L;
    for (int k = 0; k <= X; ++k) {
        if (k > 0) cum += 2.0L * expl(-static_cast<long double>(k) * k / s2);
        const long double t = floorl(two63 * (cum / S));
        if (t >= two63) break;
        T.push_back(static_cast<uint64_t>(t));
    }
    return T;
}

}  // namespace cbs
