// tcb.cu -- torus circuit bootstrapping with private functional key switching (PFKS).
//
// An LWE bit under the level-0 key s0 becomes an RGSW ciphertext under the level-1 RLWE key z1
// (CGGI 2017, circuit bootstrapping): for each output level k, a level-2 blind rotation (ring
// N2, key z2, 64-bit torus, the FFT kernel of gate.cu) of the constant test vector g_k / 2,
// plus g_k / 2 on the extracted b, gives an LWE of m g_k under z2 (the 64-bit torus keeps the
// level-2 key noise far below the output gadget; a 32-bit torus cannot: its noise floor of one
// unit, amplified by the blind rotation, already reaches ~2^-12); two private functional key
// switches (digits of the top 32 bits) turn it
// into the RGSW rows 2k (function -z1: component a carries m g_k) and 2k+1 (identity:
// component b carries m g_k).  The PFKS key of function f holds, for each input coefficient i
// (the N2 key coefficients and the constant 1 of b), digit level j and digit value v,
// RLWE_z1(f(v * y_i * 2^(32 - (j+1) * base_bits))); a switch adds the rows selected by the
// digits of (-a, b).  With base_bits * levels = 32 the digits are exact, so the switch adds
// only the key noise.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "devbuf.cuh"
#include "fft_kernels.cuh"
#include "keygen.h"
#include "torus.cuh"

namespace cbs {

// one PFKS per CTA: item = bit * levels + k, function c = blockIdx.x % 2; each thread owns the
// output coefficients tid + 256 r of the 2 * N1 words (a then b)
template <uint32_t N1>
__global__ void __launch_bounds__(256) k_tcb_pfks(const uint64_t* __restrict__ ext, const uint32_t* __restrict__ key,
                                                  uint32_t N2, uint32_t base_bits, uint32_t levels,
                                                  uint32_t* __restrict__ rgsw) {
    constexpr uint32_t R = 2 * N1 / 256;
    const uint32_t item = blockIdx.x / 2, c = blockIdx.x % 2;
    const uint32_t base = 1u << base_bits;
    const uint64_t* in = ext + static_cast<size_t>(item) * (N2 + 1);
    const size_t per_i = static_cast<size_t>(levels) * (base - 1) * 2 * N1;
    const uint32_t* kc = key + static_cast<size_t>(c) * (N2 + 1) * per_i + threadIdx.x;
    uint32_t acc[R];
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) acc[r] = 0;
    for (uint32_t i = 0; i <= N2; ++i) {
        const uint64_t x64 = (i < N2) ? 0ull - __ldg(in + i) : __ldg(in + N2);  // phase = sum x_i y_i
        const uint32_t x = static_cast<uint32_t>((x64 + (1ull << 31)) >> 32);      // top 32 bits, rounded
        const uint32_t* ki = kc + i * per_i;
        for (uint32_t j = 0; j < levels; ++j) {
            const uint32_t v = (x >> (32 - (j + 1) * base_bits)) & (base - 1);
            if (v == 0) continue;  // uniform over the CTA
            const uint32_t* row = ki + (static_cast<size_t>(j) * (base - 1) + (v - 1)) * 2 * N1;
#pragma unroll
            for (uint32_t r = 0; r < R; ++r) acc[r] += __ldg(row + r * 256);
        }
    }
    uint32_t* out = rgsw + (static_cast<size_t>(item) * 2 + c) * 2 * N1 + threadIdx.x;
#pragma unroll
    for (uint32_t r = 0; r < R; ++r) out[r * 256] = acc[r];
}

// Tiled PFKS: output rows that share the function read, for each input coefficient i and
// digit level j, the same 2^b - 1 key rows and differ only in which one their digit selects.
// A CTA owns 128 output items x 128 output words of one function: per (i, j) it stages that
// 128-word slice of the key rows in shared memory (row 0 zero, so digit 0 needs no branch)
// and each thread adds the selected rows for its 4 items x 16 words.  The slices stream
// through a 4-stage ring filled by per-thread asynchronous copies issued three slices ahead,
// and the digit words of coefficient i + 1 are loaded while coefficient i is summed, so the
// loop does not wait on memory latency.  Key traffic falls from one full key stream per
// output row to one per 128 rows; the sums are the same integers mod 2^32 as the
// one-row-per-CTA kernel.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

template <uint32_t BASE_BITS>
__global__ void __launch_bounds__(256, 2) k_tcb_pfks_tiled(const uint64_t* __restrict__ ext,
                                                          const uint32_t* __restrict__ key, uint32_t items, uint32_t N2,
                                                          uint32_t N1, uint32_t levels, uint32_t* __restrict__ rgsw) {
    constexpr uint32_t B = 1u << BASE_BITS, CT = 128, IT = 128, TPI = 4, CG = 8, STAGES = 4;
    constexpr uint32_t CHUNKS = (B - 1) * CT / 4, PER_T = (CHUNKS + 255) / 256;
    __shared__ __align__(16) uint32_t tile[STAGES][B][CT];
    const uint32_t tid = threadIdx.x, cg = tid % CG, ig = tid / CG;
    const uint32_t c0 = blockIdx.x * CT, item0 = blockIdx.y * IT + ig * TPI, fn = blockIdx.z;
    const size_t row_words = 2ull * N1, per_i = static_cast<size_t>(levels) * (B - 1) * row_words;
    const uint32_t* kf = key + static_cast<size_t>(fn) * (N2 + 1) * per_i + c0;
    const uint32_t tiles = (N2 + 1) * levels;  // slice t = i * levels + j
    if (tid < CT)
#pragma unroll
        for (uint32_t st = 0; st < STAGES; ++st) tile[st][0][tid] = 0u;
    // one commit group per slice index, issued or not, so the group count stays uniform
    auto issue = [&](uint32_t t) {
        if (t < tiles) {
            const uint32_t i = t / levels, j = t % levels;
            const uint32_t* src = kf + i * per_i + static_cast<size_t>(j) * (B - 1) * row_words;
            uint32_t (*dst)[CT] = tile[t % STAGES];
#pragma unroll
            for (uint32_t p = 0; p < PER_T; ++p) {
                const uint32_t k = tid + 256 * p;
                if (k < CHUNKS)
                    cp_async16(&dst[1 + k / (CT / 4)][(k % (CT / 4)) * 4],
                               src + (k / (CT / 4)) * row_words + (k % (CT / 4)) * 4);
            }
        }
        cp_async_commit();
    };
    // top 32 bits (rounded) of -a_i, or of b for i = N2: phase = sum x_i y_i
    auto load_x = [&](uint32_t i, uint32_t (&x)[TPI]) {
#pragma unroll
        for (uint32_t u = 0; u < TPI; ++u) {
            const uint32_t item = item0 + u;
            uint64_t x64 = 0;
            if (item < items && i <= N2) {
                const uint64_t* in = ext + static_cast<size_t>(item) * (N2 + 1);
                x64 = (i < N2) ? 0ull - __ldg(in + i) : __ldg(in + N2);
            }
            x[u] = static_cast<uint32_t>((x64 + (1ull << 31)) >> 32);
        }
    };
    uint32_t acc[TPI][16];
#pragma unroll
    for (uint32_t u = 0; u < TPI; ++u)
#pragma unroll
        for (uint32_t w = 0; w < 16; ++w) acc[u][w] = 0u;
#pragma unroll
    for (uint32_t t = 0; t < STAGES - 1; ++t) issue(t);
    uint32_t x[TPI], xn[TPI];
    load_x(0, x);
    for (uint32_t i = 0; i <= N2; ++i) {
        load_x(i + 1, xn);
        for (uint32_t j = 0; j < levels; ++j) {
            const uint32_t t = i * levels + j;
            cp_async_wait<STAGES - 2>();  // this thread's copies of slice t have landed
            __syncthreads();              // everyone's have; slice t - 1 is no longer read
            issue(t + STAGES - 1);        // into the stage slice t - 1 used
            const uint32_t sh = 32 - (j + 1) * BASE_BITS;
            const uint32_t (*cur)[CT] = tile[t % STAGES];
#pragma unroll
            for (uint32_t u = 0; u < TPI; ++u) {
                const uint32_t* row = cur[(x[u] >> sh) & (B - 1)];
#pragma unroll
                for (uint32_t q = 0; q < 4; ++q) {
                    const uint4 v = *reinterpret_cast<const uint4*>(row + 4 * (cg + CG * q));
                    acc[u][4 * q] += v.x;
                    acc[u][4 * q + 1] += v.y;
                    acc[u][4 * q + 2] += v.z;
                    acc[u][4 * q + 3] += v.w;
                }
            }
        }
#pragma unroll
        for (uint32_t u = 0; u < TPI; ++u) x[u] = xn[u];
    }
    cp_async_wait<0>();
#pragma unroll
    for (uint32_t u = 0; u < TPI; ++u) {
        const uint32_t item = item0 + u;
        if (item >= items) continue;
        uint32_t* out = rgsw + (static_cast<size_t>(item) * 2 + fn) * row_words + c0;
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q)
            *reinterpret_cast<uint4*>(out + 4 * (cg + CG * q)) =
                make_uint4(acc[u][4 * q], acc[u][4 * q + 1], acc[u][4 * q + 2], acc[u][4 * q + 3]);
    }
}

static cudaError_t tcb_pfks_launch(const uint64_t* ext, const uint32_t* key, uint32_t items, uint32_t N2, uint32_t N1,
                                   uint32_t base_bits, uint32_t levels, uint32_t* rgsw, cudaStream_t s) {
    if (base_bits == 4 && (2 * N1) % 128 == 0 && levels * base_bits <= 32) {
        const dim3 grid(2 * N1 / 128, (items + 127) / 128, 2);
        k_tcb_pfks_tiled<4><<<grid, 256, 0, s>>>(ext, key, items, N2, N1, levels, rgsw);
        return cudaGetLastError();
    }
    const unsigned grid = 2 * items;
    switch (N1) {
        case 256: k_tcb_pfks<256><<<grid, 256, 0, s>>>(ext, key, N2, base_bits, levels, rgsw); break;
        case 512: k_tcb_pfks<512><<<grid, 256, 0, s>>>(ext, key, N2, base_bits, levels, rgsw); break;
        case 1024: k_tcb_pfks<1024><<<grid, 256, 0, s>>>(ext, key, N2, base_bits, levels, rgsw); break;
        case 2048: k_tcb_pfks<2048><<<grid, 256, 0, s>>>(ext, key, N2, base_bits, levels, rgsw); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// ---- host: exact negacyclic products by a fixed binary polynomial through an FP64 FFT ----

// c = a * z (negacyclic, mod 2^32) for a torus32 polynomial a and a binary z, via the folded
// FP64 FFT of length N/2: |a * z| < 2^31 * N <= 2^43, so the rounded result is exact.
class BinaryPolyMul {
   public:
    BinaryPolyMul(const std::vector<int32_t>& z) : N_(static_cast<uint32_t>(z.size())), M_(N_ / 2) {
        const double pi = 3.141592653589793238462643383279502884;
        tw_.resize(M_ / 2 > 0 ? M_ / 2 : 1);
        for (uint32_t e = 0; e < M_ / 2; ++e) tw_[e] = std::polar(1.0, -2.0 * pi * e / M_);
        twist_.resize(M_);
        for (uint32_t e = 0; e < M_; ++e) twist_[e] = std::polar(1.0, pi * e / N_);
        zf_.resize(M_);
        for (uint32_t e = 0; e < M_; ++e) zf_[e] = std::complex<double>(z[e], z[e + M_]) * twist_[e];
        fft(zf_, false);
    }
    void mul(const uint32_t* a, uint32_t* out) const {
        std::vector<std::complex<double>> x(M_);
        for (uint32_t e = 0; e < M_; ++e)
            x[e] = std::complex<double>(static_cast<int32_t>(a[e]), static_cast<int32_t>(a[e + M_])) * twist_[e];
        fft(x, false);
        for (uint32_t e = 0; e < M_; ++e) x[e] *= zf_[e];
        fft(x, true);
        for (uint32_t e = 0; e < M_; ++e) {
            const std::complex<double> u = x[e] * std::conj(twist_[e]) / static_cast<double>(M_);
            out[e] = static_cast<uint32_t>(static_cast<uint64_t>(std::llround(u.real())));
            out[e + M_] = static_cast<uint32_t>(static_cast<uint64_t>(std::llround(u.imag())));
        }
    }

    // c = a * z mod 2^64 for a torus64 polynomial a: two exact products of its 32-bit halves
    void mul64(const uint64_t* a, uint64_t* out) const {
        std::vector<uint64_t> lo(N_), hi(N_);
        for (uint32_t e = 0; e < N_; ++e) {
            lo[e] = a[e] & 0xffffffffull;
            hi[e] = a[e] >> 32;
        }
        std::vector<int64_t> pl(N_), ph(N_);
        mul_raw(lo.data(), pl.data());
        mul_raw(hi.data(), ph.data());
        for (uint32_t e = 0; e < N_; ++e)
            out[e] = static_cast<uint64_t>(pl[e]) + (static_cast<uint64_t>(ph[e]) << 32);
    }

   private:
    // exact integer negacyclic product of v (0 <= v < 2^32) by z: |result| < 2^32 N < 2^44
    void mul_raw(const uint64_t* v, int64_t* out) const {
        std::vector<std::complex<double>> x(M_);
        for (uint32_t e = 0; e < M_; ++e)
            x[e] = std::complex<double>(static_cast<double>(v[e]), static_cast<double>(v[e + M_])) * twist_[e];
        fft(x, false);
        for (uint32_t e = 0; e < M_; ++e) x[e] *= zf_[e];
        fft(x, true);
        for (uint32_t e = 0; e < M_; ++e) {
            const std::complex<double> u = x[e] * std::conj(twist_[e]) / static_cast<double>(M_);
            out[e] = std::llround(u.real());
            out[e + M_] = std::llround(u.imag());
        }
    }
    // in-place iterative radix-2 FFT (bit-reversal first); inverse without the 1/M factor
    void fft(std::vector<std::complex<double>>& x, bool inverse) const {
        const uint32_t M = M_;
        for (uint32_t i = 1, j = 0; i < M; ++i) {
            uint32_t bit = M >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) std::swap(x[i], x[j]);
        }
        for (uint32_t len = 2; len <= M; len <<= 1) {
            const uint32_t step = M / len;
            for (uint32_t s = 0; s < M; s += len)
                for (uint32_t k = 0; k < len / 2; ++k) {
                    std::complex<double> w = tw_[k * step];
                    if (inverse) w = std::conj(w);
                    const std::complex<double> u = x[s + k], v = x[s + k + len / 2] * w;
                    x[s + k] = u + v;
                    x[s + k + len / 2] = u - v;
                }
        }
    }
    uint32_t N_, M_;
    std::vector<std::complex<double>> tw_, twist_, zf_;
};

}  // namespace cbs

// ---------------------------------------------------------------------------------------
// keys and the C ABI
// ---------------------------------------------------------------------------------------

using cbs::DevBuf;

struct cbs_tcb_context {
    cbs_tcb_params p{};
    uint32_t max_batch = 0;
    bool keys_ready = false;
    std::vector<int32_t> s0, z2, z1;
    std::vector<uint64_t> bsk2;  // level 2: 64-bit torus
    std::vector<uint32_t> pfks;
    DevBuf<double2> d_bskf, d_tab;
    DevBuf<uint32_t> d_pfks;
    DevBuf<uint64_t> d_ext;
    // grouped (multi-bit) level-2 blind rotation: mb, its keys (coefficient form), spectra
    uint32_t br_mb = 1;
    bool mb_ready = false;
    uint64_t key_seed = 0;
    std::vector<uint64_t> mbk2;
    DevBuf<double2> d_bskf_mb;
};

namespace {

using cbs::set_error;

cbs_status validate_tcb(const cbs_tcb_params& p) {
    CBS_CHECK_ARG(p.N2 >= 64 && p.N2 <= 2048 && (p.N2 & (p.N2 - 1)) == 0, "tcb: N2 must be a power of two <= 2048");
    CBS_CHECK_ARG(p.N1 >= 64 && p.N1 <= 2048 && (p.N1 & (p.N1 - 1)) == 0, "tcb: N1 must be a power of two <= 2048");
    CBS_CHECK_ARG(p.n >= 1 && p.n <= 4096, "tcb: n out of range");
    CBS_CHECK_ARG(p.bg2_bits >= 1 && p.bg2_bits <= 15 && p.l2 >= 1 && p.l2 <= 4 && p.bg2_bits * p.l2 <= 30,
                  "tcb: level-2 gadget out of range");
    CBS_CHECK_ARG(p.cb_levels >= 1 && p.cb_levels <= 8 && p.cb_bits >= 1 && p.cb_bits * p.cb_levels <= 31,
                  "tcb: output gadget out of range (cb_levels <= 8)");
    CBS_CHECK_ARG(p.pfks_base_bits >= 1 && p.pfks_base_bits <= 8 && p.pfks_base_bits * p.pfks_levels == 32,
                  "tcb: PFKS digits must cover the 32-bit torus exactly");
    CBS_CHECK_ARG(p.sigma_lwe >= 0 && p.sigma_lvl2 >= 0 && p.sigma_lvl1 >= 0 && p.sigma_lwe < 0.01 &&
                      p.sigma_lvl2 < 0.01 && p.sigma_lvl1 < 0.01,
                  "tcb: noise out of range");
    return CBS_OK;
}

size_t pfks_words(const cbs_tcb_params& p) {
    return 2ull * (p.N2 + 1) * p.pfks_levels * ((1u << p.pfks_base_bits) - 1) * 2 * p.N1;
}

uint64_t mix(uint64_t x) {  // splitmix64 finaliser: independent seeds per key row
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

void tcb_keys_host(const cbs_tcb_params& p, uint64_t seed, std::vector<int32_t>& s0, std::vector<int32_t>& z2,
                   std::vector<int32_t>& z1, std::vector<uint64_t>& bsk2, std::vector<uint32_t>* pfks) {
    const uint32_t n = p.n, N2 = p.N2, N1 = p.N1, L = p.l2, base = 1u << p.pfks_base_bits;
    cbs::Rng rng(seed ^ 0x7cb5a11c0de5eedull);
    s0.assign(n, 0);
    z2.assign(N2, 0);
    z1.assign(N1, 0);
    for (auto& v : s0) v = static_cast<int32_t>(rng.uniform(2));
    for (auto& v : z2) v = static_cast<int32_t>(rng.uniform(2));
    for (auto& v : z1) v = static_cast<int32_t>(rng.uniform(2));
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    // level-2 bootstrapping key RGSW_z2(s0_i) on the 64-bit torus: row 2k+c adds
    // s0_i * 2^(64-(k+1)*bg2_bits) to component c
    bsk2.assign(static_cast<size_t>(n) * 2 * L * 2 * N2, 0);
    {
        cbs::BinaryPolyMul mz2(z2);
        std::vector<std::thread> pool;
        const size_t rows = static_cast<size_t>(n) * 2 * L;
        for (unsigned th = 0; th < nth; ++th)
            pool.emplace_back([&, th] {
                std::vector<uint64_t> prod(N2);
                for (size_t r = th; r < rows; r += nth) {
                    cbs::Rng rr(mix(seed * 4 + 1) ^ mix(r));
                    uint64_t* ra = bsk2.data() + r * 2 * N2;
                    uint64_t* rb = ra + N2;
                    for (uint32_t e = 0; e < N2; ++e) ra[e] = rr.next();
                    mz2.mul64(ra, prod.data());
                    for (uint32_t e = 0; e < N2; ++e)
                        rb[e] = prod[e] + static_cast<uint64_t>(
                                              std::llround(rr.gaussian() * p.sigma_lvl2 * 18446744073709551616.0));
                    const uint32_t i = static_cast<uint32_t>(r / (2 * L)), row = static_cast<uint32_t>(r % (2 * L));
                    const uint32_t k = row / 2, c = row % 2;
                    (c ? rb : ra)[0] += static_cast<uint64_t>(s0[i]) << (64 - (k + 1) * p.bg2_bits);
                }
            });
        for (auto& t : pool) t.join();
    }
    if (!pfks) return;
    // PFKS keys [f][i][j][v-1] = RLWE_z1(f(v * y_i * g_j)), f = 0: x -> -x z1, f = 1: identity
    pfks->assign(pfks_words(p), 0);
    cbs::BinaryPolyMul mz1(z1);
    const size_t rows = 2ull * (N2 + 1) * p.pfks_levels * (base - 1);
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th)
        pool.emplace_back([&, th] {
            std::vector<uint32_t> prod(N1);
            for (size_t r = th; r < rows; r += nth) {
                cbs::Rng rr(mix(seed * 4 + 2) ^ mix(r));
                size_t t = r;
                const uint32_t v = static_cast<uint32_t>(t % (base - 1)) + 1;
                t /= (base - 1);
                const uint32_t j = static_cast<uint32_t>(t % p.pfks_levels);
                t /= p.pfks_levels;
                const uint32_t i = static_cast<uint32_t>(t % (N2 + 1));
                const uint32_t f = static_cast<uint32_t>(t / (N2 + 1));
                const uint32_t y = (i < N2) ? static_cast<uint32_t>(z2[i]) : 1u;
                const uint32_t m0 = v * y * (1u << (32 - (j + 1) * p.pfks_base_bits));
                uint32_t* ra = pfks->data() + r * 2 * N1;
                uint32_t* rb = ra + N1;
                for (uint32_t e = 0; e < N1; ++e) ra[e] = static_cast<uint32_t>(rr.next());
                mz1.mul(ra, prod.data());
                for (uint32_t e = 0; e < N1; ++e) rb[e] = prod[e] + cbs::torus_noise(rr, p.sigma_lvl1);
                if (f == 1) {
                    rb[0] += m0;
                } else {
                    for (uint32_t e = 0; e < N1; ++e) rb[e] -= m0 * static_cast<uint32_t>(z1[e]);
                }
            }
        });
    for (auto& t : pool) t.join();
}

// Grouped level-2 keys RGSW_z2(prod_{i in S} s0_i) on the 64-bit torus for every non-empty
// subset S of each group of mb coefficients (row 2k + c adds the product times
// 2^(64 - (k+1) bg2) to component c); one generator per row.
void tcb_mb_keys_host(const cbs_tcb_params& p, const std::vector<int32_t>& s0, const std::vector<int32_t>& z2,
                      uint32_t mb, uint64_t seed, std::vector<uint64_t>& out) {
    const uint32_t n = p.n, N2 = p.N2, L = p.l2, K = cbs::mb_subsets(mb), groups = (n + mb - 1) / mb;
    const size_t rows = static_cast<size_t>(groups) * K * 2 * L;
    out.assign(rows * 2 * N2, 0);
    cbs::BinaryPolyMul mz2(z2);
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th)
        pool.emplace_back([&, th] {
            std::vector<uint64_t> prod(N2);
            for (size_t r = th; r < rows; r += nth) {
                cbs::Rng rr(mix(seed * 4 + 3) ^ mix(r));
                uint64_t* ra = out.data() + r * 2 * N2;
                uint64_t* rb = ra + N2;
                for (uint32_t e = 0; e < N2; ++e) ra[e] = rr.next();
                mz2.mul64(ra, prod.data());
                for (uint32_t e = 0; e < N2; ++e)
                    rb[e] = prod[e] + static_cast<uint64_t>(
                                          std::llround(rr.gaussian() * p.sigma_lvl2 * 18446744073709551616.0));
                const uint32_t g = static_cast<uint32_t>(r / (K * 2 * L));
                const uint32_t kk = static_cast<uint32_t>((r / (2 * L)) % K), row = static_cast<uint32_t>(r % (2 * L));
                const uint32_t mask = cbs::mb_subset_mask(mb, kk);
                uint64_t prodb = 1;
                for (uint32_t i = 0; i < mb; ++i)
                    if (mask & (1u << i)) prodb &= (g * mb + i < n) ? static_cast<uint64_t>(s0[g * mb + i]) : 0u;
                (row % 2 ? rb : ra)[0] += prodb << (64 - (row / 2 + 1) * p.bg2_bits);
            }
        });
    for (auto& t : pool) t.join();
}

cbs_status tcb_prepare_mb(cbs_tcb_context* ctx) {
    if (ctx->br_mb <= 1 || ctx->mb_ready || !ctx->keys_ready) return CBS_OK;
    std::vector<double2> spec;
    try {
        tcb_mb_keys_host(ctx->p, ctx->s0, ctx->z2, ctx->br_mb, ctx->key_seed, ctx->mbk2);
        cbs::torus_keys_to_fft(ctx->p.N2, ctx->mbk2.data(), ctx->mbk2.size() / ctx->p.N2, spec);
    } catch (const std::exception& e) {
        set_error(std::string("tcb multi-bit keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    CBS_CUDA_TRY(ctx->d_bskf_mb.upload(spec.data(), spec.size(), nullptr));
    CBS_CUDA_TRY(cudaStreamSynchronize(nullptr));
    ctx->mb_ready = true;
    return CBS_OK;
}

}  // namespace

extern "C" {

cbs_status cbs_tcb_params_default(cbs_tcb_params* out) {
    CBS_CHECK_ARG(out, "tcb_params_default: null argument");
    out->n = 630;
    out->N2 = 2048;
    out->bg2_bits = 9;
    out->l2 = 3;
    out->N1 = 1024;
    out->cb_bits = 6;
    out->cb_levels = 3;
    out->pfks_base_bits = 4;
    out->pfks_levels = 8;
    out->sigma_lwe = std::ldexp(1.0, -15);
    out->sigma_lvl2 = std::ldexp(1.0, -44);
    out->sigma_lvl1 = std::ldexp(1.0, -25);
    return CBS_OK;
}

cbs_status cbs_tcb_context_create(const cbs_tcb_params* params, uint32_t max_batch, cbs_tcb_context** out) {
    CBS_CHECK_ARG(params && out, "tcb_context_create: null argument");
    *out = nullptr;
    if (cbs_status st = validate_tcb(*params)) return st;
    CBS_CHECK_ARG(params->N2 == 1024 || params->N2 == 2048,
                  "tcb_context_create: the device blind rotation needs N2 of 1024 or 2048");
    CBS_CHECK_ARG(params->N1 >= 256, "tcb_context_create: the device PFKS needs N1 >= 256");
    CBS_CHECK_ARG(max_batch >= 1 && max_batch <= (1u << 20), "tcb_context_create: max_batch out of range");
    auto* c = new (std::nothrow) cbs_tcb_context();
    if (!c) {
        set_error("tcb_context_create: host allocation failed");
        return CBS_ERR_OOM;
    }
    std::unique_ptr<cbs_tcb_context> guard(c);
    c->p = *params;
    c->max_batch = max_batch;
    CBS_CUDA_TRY(c->d_ext.alloc(static_cast<size_t>(max_batch) * params->cb_levels * (params->N2 + 1)));
    *out = guard.release();
    return CBS_OK;
}

cbs_status cbs_tcb_context_destroy(cbs_tcb_context* ctx) {
    delete ctx;
    return CBS_OK;
}

cbs_status cbs_tcb_generate_keys_host(const cbs_tcb_params* params, uint64_t seed, int32_t* s0, int32_t* z2,
                                      int32_t* z1, uint64_t* bsk2, uint32_t* pfks) {
    CBS_CHECK_ARG(params, "tcb_generate_keys_host: null params");
    if (cbs_status st = validate_tcb(*params)) return st;
    std::vector<int32_t> a, b, c;
    std::vector<uint64_t> k2;
    std::vector<uint32_t> kp;
    tcb_keys_host(*params, seed, a, b, c, k2, pfks ? &kp : nullptr);
    if (s0) std::copy(a.begin(), a.end(), s0);
    if (z2) std::copy(b.begin(), b.end(), z2);
    if (z1) std::copy(c.begin(), c.end(), z1);
    if (bsk2) std::copy(k2.begin(), k2.end(), bsk2);
    if (pfks) std::copy(kp.begin(), kp.end(), pfks);
    return CBS_OK;
}

cbs_status cbs_tcb_keygen(cbs_tcb_context* ctx, uint64_t seed) {
    CBS_CHECK_ARG(ctx, "tcb_keygen: null context");
    const cbs_tcb_params& p = ctx->p;
    tcb_keys_host(p, seed, ctx->s0, ctx->z2, ctx->z1, ctx->bsk2, &ctx->pfks);
    std::vector<double2> bskf, tab;
    cbs::torus_keys_to_fft(p.N2, ctx->bsk2.data(), ctx->bsk2.size() / p.N2, bskf);
    cbs::fft_tables_host(p.N2, tab);
    CBS_CUDA_TRY(ctx->d_bskf.upload(bskf.data(), bskf.size(), nullptr));
    CBS_CUDA_TRY(ctx->d_tab.upload(tab.data(), tab.size(), nullptr));
    CBS_CUDA_TRY(ctx->d_pfks.upload(ctx->pfks.data(), ctx->pfks.size(), nullptr));
    CBS_CUDA_TRY(cudaStreamSynchronize(nullptr));
    ctx->keys_ready = true;
    ctx->key_seed = seed;
    ctx->mb_ready = false;
    return tcb_prepare_mb(ctx);
}

cbs_status cbs_tcb_set_multibit(cbs_tcb_context* ctx, uint32_t mb) {
    CBS_CHECK_ARG(ctx, "tcb_set_multibit: null context");
    CBS_CHECK_ARG(mb >= 1 && mb <= 3, "tcb_set_multibit: mb must be 1, 2 or 3");
    if (mb != ctx->br_mb) {
        ctx->br_mb = mb;
        ctx->mb_ready = false;
        ctx->mbk2.clear();
        ctx->d_bskf_mb.reset();
    }
    return tcb_prepare_mb(ctx);
}

cbs_status cbs_tcb_export_mb_bsk(const cbs_tcb_context* ctx, uint64_t* out, size_t* words) {
    CBS_CHECK_ARG(ctx && words, "tcb_export_mb_bsk: null argument");
    if (ctx->br_mb <= 1 || !ctx->mb_ready) {
        set_error("tcb_export_mb_bsk: no grouped keys (select mb > 1 after cbs_tcb_keygen)");
        return CBS_ERR_NOT_READY;
    }
    *words = ctx->mbk2.size();
    if (out) std::copy(ctx->mbk2.begin(), ctx->mbk2.end(), out);
    return CBS_OK;
}

cbs_status cbs_tcb_export_keys(const cbs_tcb_context* ctx, int32_t* s0, int32_t* z2, int32_t* z1, uint64_t* bsk2,
                               uint32_t* pfks) {
    CBS_CHECK_ARG(ctx, "tcb_export_keys: null context");
    if (!ctx->keys_ready) {
        set_error("tcb_export_keys: no keys (call cbs_tcb_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    if (s0) std::copy(ctx->s0.begin(), ctx->s0.end(), s0);
    if (z2) std::copy(ctx->z2.begin(), ctx->z2.end(), z2);
    if (z1) std::copy(ctx->z1.begin(), ctx->z1.end(), z1);
    if (bsk2) std::copy(ctx->bsk2.begin(), ctx->bsk2.end(), bsk2);
    if (pfks) std::copy(ctx->pfks.begin(), ctx->pfks.end(), pfks);
    return CBS_OK;
}

cbs_status cbs_tcb_encrypt_bits(const cbs_tcb_context* ctx, const uint8_t* h_bits, uint32_t count, uint64_t seed,
                                uint32_t* h_a, uint32_t* h_b) {
    CBS_CHECK_ARG(ctx && h_bits && h_a && h_b, "tcb_encrypt_bits: null argument");
    if (!ctx->keys_ready) {
        set_error("tcb_encrypt_bits: no keys (call cbs_tcb_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    cbs::Rng rng(seed);
    const uint32_t n = ctx->p.n;
    for (uint32_t k = 0; k < count; ++k) {
        // bit m -> phase m/4 - 1/8 (i.e. -1/8 or +1/8): the blind rotation's sign then gives +-g/2
        uint32_t b = (h_bits[k] ? (1u << 29) : (0u - (1u << 29))) + cbs::torus_noise(rng, ctx->p.sigma_lwe);
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t a = static_cast<uint32_t>(rng.next());
            h_a[static_cast<size_t>(k) * n + j] = a;
            if (ctx->s0[j]) b += a;
        }
        h_b[k] = b;
    }
    return CBS_OK;
}

cbs_status cbs_tcb_circuit_bootstrap_device(cbs_tcb_context* ctx, const uint32_t* d_a, const uint32_t* d_b,
                                            uint32_t count, uint64_t* d_ext, uint32_t* d_rgsw, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && d_a && d_b && d_rgsw, "tcb_circuit_bootstrap: null argument");
    if (!ctx->keys_ready) {
        set_error("tcb_circuit_bootstrap: no keys (call cbs_tcb_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    if (count == 0) return CBS_OK;
    if (count > ctx->max_batch) {
        set_error("tcb_circuit_bootstrap: count above the context's max_batch");
        return CBS_ERR_SHAPE_MISMATCH;
    }
    const cbs_tcb_params& p = ctx->p;
    if (ctx->br_mb > 1 && !ctx->mb_ready) {
        set_error("tcb_circuit_bootstrap: grouped keys are not prepared");
        return CBS_ERR_NOT_READY;
    }
    cbs::GateArgs a{};
    a.gate = -1;
    a.a1 = d_a;
    a.b1 = d_b;
    a.n = p.n;
    a.levels = p.l2;
    a.bg_bits = p.bg2_bits;
    a.bskf = ctx->br_mb > 1 ? ctx->d_bskf_mb.p : ctx->d_bskf.p;
    a.mb = ctx->br_mb;
    a.tab = ctx->d_tab.p;
    a.ext = d_ext ? d_ext : ctx->d_ext.p;
    a.items = count * p.cb_levels;
    a.levels_tv = p.cb_levels;
    for (uint32_t k = 0; k < p.cb_levels; ++k) {
        const uint64_t half_g = 1ull << (64 - (k + 1) * p.cb_bits - 1);
        a.mu[k] = half_g;     // sign bootstrap to +-g_k / 2 (64-bit torus)
        a.b_add[k] = half_g;  // +g_k / 2: m g_k
    }
    CBS_CUDA_TRY(cbs::gate_blind_rotate64(a, p.N2, a.items, stream));
    CBS_CUDA_TRY(cbs::tcb_pfks_launch(static_cast<const uint64_t*>(a.ext), ctx->d_pfks.p, a.items, p.N2, p.N1,
                                      p.pfks_base_bits, p.pfks_levels, d_rgsw, stream));
    return CBS_OK;
}

}  // extern "C"
