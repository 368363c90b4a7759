// extract_kernels.cu -- sample extraction + LWE key switch, and the AES state glue kernels.
//
// k_extract_keyswitch follows the contract of examples/aes_gpu_ks.cuh:538-607
// (kernel_SampleExtractKeySwitchToLWE): for output bit t, extract coefficient idx of RLWE
// word w (a'_j = a[idx-j], or -a[N+idx-j]), switch each coefficient Q -> qKS with the same
// FP64 round-to-nearest expression (aes_gpu_ks.cuh:388-394), key-switch N -> n with two
// base-2^k digits against the u16 key, and map qKS -> q (exact scale, or round-half-up
// division when q is not a multiple of qKS, aes_gpu_ks.cuh:431-440).  One CTA per output
// bit, 4 outputs per thread; the mod-switched mask is staged in shared memory and
// consecutive threads read consecutive 8-byte segments of a key row.
#include "common.cuh"
#include "extract_kernels.cuh"

namespace cbs {

__device__ __forceinline__ uint32_t ms_pow2(uint64_t v, double q_over_Q, uint32_t mask) {
    return static_cast<uint32_t>(__double2uint_rn(static_cast<double>(v) * q_over_Q)) & mask;
}

__device__ __forceinline__ uint64_t qks_to_q(uint32_t v, uint64_t scale, uint32_t qks, uint64_t q) {
    if (scale) return static_cast<uint64_t>(v) * scale;
    const unsigned __int128 x = static_cast<unsigned __int128>(v) * q + (qks >> 1);
    return static_cast<uint64_t>(x / qks);
}

// One CTA per output bit: the mod-switched mask (N u16) is staged in shared memory once, and
// each thread accumulates 4 consecutive outputs from one 8-byte load per key row (rows padded
// to a multiple of 4 words), unrolled so that 16 independent loads are in flight.
constexpr uint32_t kExtractThreads = 256;

__global__ void __launch_bounds__(kExtractThreads) k_extract_keyswitch(const ExtractArgs a) {
    extern __shared__ uint16_t s_a[];  // [N]
    const uint32_t t = blockIdx.x;
    const uint32_t outlen = a.n + 1, stride = a.ksk_stride;
    const uint32_t info = __ldg(a.info + t);
    const uint32_t word = info >> 16, idx = info & 0xFFFFu;
    const uint64_t* aw = a.words + static_cast<size_t>(word) * 2 * a.N;
    const uint64_t* bw = aw + a.N;
    for (uint32_t c = threadIdx.x; c < a.N; c += blockDim.x) {
        uint64_t v;
        if (c <= idx) {
            v = aw[idx - c];
        } else {
            const uint64_t x = aw[a.N + idx - c];
            v = x ? a.Q - x : 0;
        }
        s_a[c] = static_cast<uint16_t>(ms_pow2(v, a.q_over_Q, a.mask));
    }
    __syncthreads();
    const uint32_t bmask = a.base_ks - 1;
    const size_t stride_i = static_cast<size_t>(a.base_ks) * stride;
    const size_t stride_j = static_cast<size_t>(a.N) * stride_i;
    for (uint32_t q = threadIdx.x; 4 * q < outlen; q += blockDim.x) {
        uint32_t acc0 = 0, acc1 = 0, acc2 = 0, acc3 = 0;
        const uint16_t* k0 = a.ksk + 4 * q;
        const uint16_t* k1 = k0 + stride_j;
#pragma unroll 8
        for (uint32_t j = 0; j < a.N; ++j) {
            const uint32_t ai = s_a[j];
            const uint32_t d0 = ai & bmask, d1 = (ai >> a.base_log2) & bmask;
            const uint2 u = __ldg(reinterpret_cast<const uint2*>(k0 + d0 * stride));
            const uint2 v = __ldg(reinterpret_cast<const uint2*>(k1 + d1 * stride));
            acc0 -= (u.x & 0xffffu) + (v.x & 0xffffu);
            acc1 -= (u.x >> 16) + (v.x >> 16);
            acc2 -= (u.y & 0xffffu) + (v.y & 0xffffu);
            acc3 -= (u.y >> 16) + (v.y >> 16);
            k0 += stride_i;
            k1 += stride_i;
        }
        const uint32_t accs[4] = {acc0, acc1, acc2, acc3};
#pragma unroll
        for (uint32_t w = 0; w < 4; ++w) {
            const uint32_t k = 4 * q + w;
            if (k > a.n) break;
            uint32_t accv = accs[w];
            if (k == a.n) accv += ms_pow2(bw[idx], a.q_over_Q, a.mask);
            const uint64_t val = qks_to_q(accv & a.mask, a.scale, a.qks, a.q_lwe);
            if (k == a.n) a.out_b[t] = val;
            else a.out_a[static_cast<size_t>(t) * a.out_stride + k] = val;
        }
    }
}

cudaError_t launch_extract_keyswitch(const ExtractArgs& a, uint32_t count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    if (a.ksk_stride % 4 != 0 || a.ksk_stride < a.n + 1) return cudaErrorInvalidValue;
    // one thread per 4 outputs (158 at n = 630), rounded to whole warps
    const uint32_t quads = a.ksk_stride / 4;
    const uint32_t threads = quads >= kExtractThreads ? kExtractThreads : ((quads + 31) / 32) * 32;
    k_extract_keyswitch<<<count, threads, a.N * sizeof(uint16_t), s>>>(a);
    return cudaGetLastError();
}

// state init (gpu_lut.cuh:430 kernel_InitLWEStateFromRoundKey): bit t of block
// t/128 = Enc(rk0 bit) + public counter bit * q/2
__global__ void k_init_state(uint64_t* out_a, uint64_t* out_b, const uint64_t* rk_a, const uint64_t* rk_b,
                             const uint8_t* bits, uint64_t half, uint64_t q, uint32_t n, uint32_t total) {
    const size_t tid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t outlen = n + 1;
    if (tid >= static_cast<size_t>(total) * outlen) return;
    const uint32_t t = static_cast<uint32_t>(tid / outlen);
    const uint32_t k = static_cast<uint32_t>(tid - static_cast<size_t>(t) * outlen);
    const uint32_t bi = t & 127u;
    if (k == n) {
        uint64_t v = rk_b[bi];
        if (bits[t]) {
            v += half;
            if (v >= q) v -= q;
        }
        out_b[t] = v;
    } else {
        out_a[static_cast<size_t>(t) * n + k] = rk_a[static_cast<size_t>(bi) * n + k];
    }
}

cudaError_t launch_init_state(uint64_t* out_a, uint64_t* out_b, const uint64_t* rk_a, const uint64_t* rk_b,
                              const uint8_t* bits, uint64_t half, uint64_t q, uint32_t n, uint32_t total,
                              cudaStream_t s) {
    const size_t work = static_cast<size_t>(total) * (n + 1);
    if (!work) return cudaSuccess;
    k_init_state<<<static_cast<unsigned>((work + 255) / 256), 256, 0, s>>>(out_a, out_b, rk_a, rk_b, bits, half, q, n,
                                                                           total);
    return cudaGetLastError();
}

// transciphering proper (main.cu:1569-1582, EvalAddConstEq(ct, q/2) per set bit): the
// keystream LWE of bit t gains q/2 where bit t of the public AES-CTR ciphertext is 1, so b
// then encrypts the plaintext bit.  bytes [total / 8], bit t = byte t/8, bit t%8 (LSB first).
__global__ void k_add_public_bits(uint64_t* b, const uint8_t* bytes, uint64_t half, uint64_t q, uint32_t total) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    if ((bytes[t >> 3] >> (t & 7u)) & 1u) {
        uint64_t v = b[t] + half;
        if (v >= q) v -= q;
        b[t] = v;
    }
}

cudaError_t launch_add_public_bits(uint64_t* b, const uint8_t* bytes, uint64_t half, uint64_t q, uint32_t total,
                                   cudaStream_t s) {
    if (!total) return cudaSuccess;
    k_add_public_bits<<<(total + 255) / 256, 256, 0, s>>>(b, bytes, half, q, total);
    return cudaGetLastError();
}

// AES word assembly: out column c of block b = sum over rows of the LUT of byte (row, c+row)
// plus the round-key word (the reference's fused final add, gpu_lut.cuh:1305-1370, and
// kernel_RLWE_AddWords4Inplace_Blocks, main.cu:1516-1523).  lut_out [blocks][16][2][N] with
// LUT index row*4 + col; rk [4][2][N]; words [blocks][4][2][N].  NTT domain throughout.
__global__ void k_assemble_words(uint64_t* words, const uint64_t* lut_out, const uint64_t* rk, uint64_t Q, uint32_t N,
                                 uint32_t blocks) {
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t per_block = 4ull * 2 * N;
    if (idx >= per_block * blocks) return;
    const uint32_t b = static_cast<uint32_t>(idx / per_block);
    const size_t rem = idx - static_cast<size_t>(b) * per_block;
    const uint32_t c = static_cast<uint32_t>(rem / (2ull * N));
    const size_t pc = rem - static_cast<size_t>(c) * 2 * N;  // poly * N + coeff
    uint64_t acc = rk[static_cast<size_t>(c) * 2 * N + pc];
#pragma unroll
    for (uint32_t row = 0; row < 4; ++row) {
        const uint32_t col = (c + row) & 3u;
        const uint64_t v = lut_out[((static_cast<size_t>(b) * 16 + row * 4 + col) * 2) * N + pc];
        acc += v;
        if (acc >= Q) acc -= Q;
    }
    words[idx] = acc;
}

cudaError_t launch_assemble_words(uint64_t* words, const uint64_t* lut_out, const uint64_t* rk, uint64_t Q, uint32_t N,
                                  uint32_t blocks, cudaStream_t s) {
    const size_t work = static_cast<size_t>(blocks) * 8 * N;
    if (!work) return cudaSuccess;
    k_assemble_words<<<static_cast<unsigned>((work + 255) / 256), 256, 0, s>>>(words, lut_out, rk, Q, N, blocks);
    return cudaGetLastError();
}

}  // namespace cbs
