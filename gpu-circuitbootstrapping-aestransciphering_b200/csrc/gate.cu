// gate.cu -- gate bootstrapping on the 32-bit torus with the FP64 FFT external product.
//
// The path of GPUBinFHEContext::BatchGPUEvalBinGate (bitwise/src/binfhe-base-scheme-batch.cu:
// 82-200): linear gate combination of two LWE ciphertexts, modulus switch to 2N, GINX blind
// rotation of the test vector 1/8 (binfhe-base-scheme-batch.cu:16-74, bitwise/src/
// rgsw-acc-batch.cu), sample extract of coefficient 0 and the LWE key switch N -> n
// (binfhe-base-scheme-batch.cu:119-185).  The reference runs the external product through
// cuFFTDx in FP64 (bitwise/src/fft.cu:3614-3883); here it is the register-blocked FFT of
// fft_core.cuh.  Parameters are the torus form of the configuration (32-bit torus, binary
// secrets), so every residue is a uint32 and every modular reduction is the natural wrap.
// Products of 7-bit digits by 32-bit keys over N <= 2048 stay below 2^51 in magnitude, so
// rounding the FFT output recovers the exact integer product: the results equal exact
// integer arithmetic (checked bit for bit against the oracle).
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "devbuf.cuh"
#include "fft_core.cuh"
#include "fft_kernels.cuh"
#include "fft_ops.cuh"
#include "keygen.h"
#include "torus.cuh"

namespace cbs {

// request holding ragged item `item` (binary search over the offsets)
__device__ __forceinline__ uint32_t gate_req_of(const GateReq* reqs, uint32_t num, uint32_t item) {
    uint32_t lo = 0, hi = num;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (__ldg(&reqs[mid].offset) <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t gate_a(int gate, uint32_t x1, uint32_t x2) {
    const uint32_t s = x1 + x2;
    switch (gate) {
        case 0: case 1: return s;
        case 2: case 3: return 0u - s;
        case 4: return 2u * s;
        case 5: return 0u - 2u * s;
        default: return x1;
    }
}

__device__ __forceinline__ uint32_t gate_b(int gate, uint32_t x1, uint32_t x2) {
    const uint32_t e8 = 1u << 29, e4 = 1u << 30, s = x1 + x2;
    switch (gate) {
        case 0: return e8 + s;
        case 1: return (0u - e8) + s;
        case 2: return (0u - e8) - s;
        case 3: return e8 - s;
        case 4: return e4 + 2u * s;
        case 5: return (0u - e4) - 2u * s;
        default: return x1;
    }
}

template <int LOGM, class C>
__device__ __forceinline__ C gate_twist(const C* tws, int j, uint32_t e) {
    if (j < 4) return tws[e];
    const C t = tws[(1u << LOGM) - e];
    C r;
    r.x = t.y;
    r.y = t.x;
    return r;
}

// the torus value of the FP64 result v of an integer-valued product: exact for 32-bit
// tori (|v| < 2^52); for 64-bit tori v carries FP64 rounding, reduced mod 2^64 exactly
template <typename TT>
__device__ __forceinline__ TT to_torus(double v);
template <>
__device__ __forceinline__ uint32_t to_torus<uint32_t>(double v) {
    return static_cast<uint32_t>(static_cast<uint64_t>(__double2ll_rn(v)));
}
template <>
__device__ __forceinline__ uint64_t to_torus<uint64_t>(double v) {
    const double k = rint(v * 0x1p-64);
    double r = fma(-k, 0x1p64, v);  // exact: v - k 2^64, |r| <= 2^63
    if (r >= 0x1p63) r -= 0x1p64;
    return static_cast<uint64_t>(__double2ll_rn(r));
}

template <int LOGN>
struct GateCfg {
    static constexpr uint32_t T = (1u << LOGN) / 8;
    static constexpr int MIN_BLOCKS = LOGN <= 10 ? 4 : 2;
};

// One CTA of two halves (M/8 threads each) per ciphertext; half h owns accumulator component
// h (0: a, 1: b), all in shared memory.  Same step structure as k_blind_rotate_fft: digits of
// the own component, forward FFT + products against both key columns per digit, swap of
// partial sums, inverse FFT, rounding to the torus, rotate-add acc += (X^a - 1) t in place.
template <int LOGN, typename TT>
__global__ void __launch_bounds__(GateCfg<LOGN>::T, GateCfg<LOGN>::MIN_BLOCKS) k_gate_blind_rotate(const GateArgs a) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, T = 2 * TH, TWO_N = 2 * N;
    constexpr uint32_t SH = 32 - (LOGN + 1);  // torus -> Z_2N
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    double2* fs = reinterpret_cast<double2*>(smem);                 // [2][M]
    double2* tab = fs + 2 * M;                                      // FftTab<LOGM>
    TT* acc = reinterpret_cast<TT*>(tab + Tb::size());             // [2][N] torus values
    uint32_t* dig = reinterpret_cast<uint32_t*>(acc + 2 * N);      // [2][levels][M] packed pairs
    const double2* tws = tab + Tb::twist_off();
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const uint32_t h = tid / TH, ht = tid % TH;
    TT* my_acc = acc + h * N;
    double2* my_fs = fs + h * M;
    const uint32_t levels = a.levels, bg = a.bg_bits;
    constexpr uint32_t W = 8 * sizeof(TT);  // torus width: 32 or 64 bits
    TT off = TT(1) << (W - levels * bg - 1);  // rounding of the dropped bits
    for (uint32_t k = 0; k < levels; ++k) off += (TT(1) << (bg - 1)) << (W - (k + 1) * bg);
    auto half_bar = [h]() {
        if (h == 0) asm volatile("bar.sync 1, %0;" ::"n"(TH) : "memory");
        else asm volatile("bar.sync 2, %0;" ::"n"(TH) : "memory");
    };
    auto ms = [](uint32_t x) { return ((x + (1u << (SH - 1))) >> SH) & (TWO_N - 1); };

    for (uint32_t i = tid; i < Tb::size(); i += T) tab[i] = a.tab[i];
    const uint32_t l2 = 2 * levels;
    for (uint32_t item = ct; item < a.items; item += gridDim.x) {
        const uint32_t* a1;
        const uint32_t* a2;
        uint32_t b;
        if (a.reqs) {  // ragged: one bootstrap of request r
            const GateReq& rq = a.reqs[gate_req_of(a.reqs, a.num_reqs, item)];
            const uint32_t k = item - rq.offset;
            a1 = rq.a + static_cast<size_t>(k) * a.n;
            a2 = a1;
            b = rq.b[k];
        } else {
            const uint32_t in = item / a.levels_tv;
            a1 = a.a1 + static_cast<size_t>(in) * a.n;
            a2 = a.a2 ? a.a2 + static_cast<size_t>(in) * a.n : a1;
            b = gate_b(a.gate, a.b1[in], a.b2 ? a.b2[in] : 0u);
        }
        const TT mu = static_cast<TT>(a.mu[item % a.levels_tv]), b_add = static_cast<TT>(a.b_add[item % a.levels_tv]);
        {
            const uint32_t bt = ms(b);
            for (uint32_t i = tid; i < N; i += T) {
                acc[i] = 0;
                const uint32_t sp = (i + bt) & (TWO_N - 1);
                const TT tv = a.tv ? static_cast<TT>(__ldg(a.tv + (sp & (N - 1)))) : mu;
                acc[N + i] = sp < N ? tv : TT(0) - tv;
            }
        }
        __syncthreads();

        for (uint32_t step = 0; step < a.n; ++step) {
            const uint32_t at = ms(a.reqs ? __ldg(a1 + step) : gate_a(a.gate, __ldg(a1 + step), __ldg(a2 + step)));
            if (at == 0) continue;  // X^0 - 1 = 0: the step adds nothing (uniform over the CTA)
            for (uint32_t e = ht; e < M; e += TH) {
                const TT wr = my_acc[e] + off, wi = my_acc[e + M] + off;
                uint32_t* dst = dig + h * levels * M + e;
                for (uint32_t k = 0; k < levels; ++k) {
                    const uint32_t s = W - (k + 1) * bg, mask = (1u << bg) - 1, half = 1u << (bg - 1);
                    const int32_t dr = static_cast<int32_t>((wr >> s) & mask) - static_cast<int32_t>(half);
                    const int32_t di = static_cast<int32_t>((wi >> s) & mask) - static_cast<int32_t>(half);
                    dst[k * M] = (static_cast<uint32_t>(dr) & 0xffffu) | (static_cast<uint32_t>(di) << 16);
                }
            }
            half_bar();
            const double2* ek = a.bskf + static_cast<size_t>(step) * l2 * 2 * M + ht;
            double2 y0[8], y1[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) y0[j] = y1[j] = make_double2(0.0, 0.0);
            for (uint32_t d = 0; d < levels; ++d) {
                const uint32_t* dsrc = dig + (h * levels + d) * M;
                double2 x[8];
                fft_forward_to_regs<LOGM>(
                    my_fs, ht, tab,
                    [&](int j, uint32_t e) {
                        const uint32_t v = dsrc[e];
                        const double re = static_cast<double>(static_cast<int16_t>(v & 0xffffu));
                        const double im = static_cast<double>(static_cast<int16_t>(v >> 16));
                        return cmul(make_double2(re, im), gate_twist<LOGM>(tws, j, e));
                    },
                    x, half_bar);
                const double2* k0 = ek + static_cast<size_t>(2 * d + h) * 2 * M;
                const double2* k1 = k0 + M;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    cfma(y0[j], x[j], __ldg(k0 + j * TH));
                    cfma(y1[j], x[j], __ldg(k1 + j * TH));
                }
                half_bar();
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) my_fs[cswz(8 * ht + j)] = h ? y0[j] : y1[j];
            __syncthreads();
            {
                const double2* take = fs + (1 - h) * M;
#pragma unroll
                for (int j = 0; j < 8; ++j) y0[j] = cadd(h ? y1[j] : y0[j], take[cswz(8 * ht + j)]);
            }
            __syncthreads();
            TT tre[8], tim[8];
            constexpr double inv_m = 1.0 / M;
            fft_inverse_from_regs<LOGM>(
                my_fs, ht, tab, y0,
                [&](int j, uint32_t e, double2 v) {
                    const double2 u = cmulc(v, gate_twist<LOGM>(tws, j, e));
                    tre[j] = to_torus<TT>(u.x * inv_m);
                    tim[j] = to_torus<TT>(u.y * inv_m);
                },
                half_bar);
            half_bar();
            TT* tsm = reinterpret_cast<TT*>(my_fs);  // N values (the buffer holds 16 M = 8 N bytes)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                tsm[ht + j * TH] = tre[j];
                tsm[ht + j * TH + M] = tim[j];
            }
            half_bar();
#pragma unroll 4
            for (uint32_t k = 0; k < N / TH; ++k) {
                const uint32_t i = ht + k * TH;
                const uint32_t s = (i + TWO_N - at) & (TWO_N - 1);
                const TT v = (s < N) ? tsm[s] : TT(0) - tsm[s - N];
                my_acc[i] += v - tsm[i];
            }
        }
        __syncthreads();
        // sample extract of coefficient 0: a'_0 = a_0, a'_i = -a_(N-i), b' = b_0
        TT* out = reinterpret_cast<TT*>(a.ext) + static_cast<size_t>(item) * (N + 1);
        for (uint32_t i = tid; i <= N; i += T) {
            TT v;
            if (i == N) v = acc[N] + b_add;
            else if (i == 0) v = acc[0];
            else v = TT(0) - acc[N - i];
            out[i] = v;
        }
        __syncthreads();  // acc is re-initialised by the next item
    }
}

// inputs of item `item` of a blind-rotation launch: the LWE rows a1 and a2 (a2 = a1 outside
// gate mode) and the combined b
__device__ __forceinline__ void gate_item_inputs(const GateArgs& a, uint32_t item, const uint32_t*& a1,
                                                 const uint32_t*& a2, uint32_t& b) {
    if (a.reqs) {  // ragged: one bootstrap of request r
        const GateReq& rq = a.reqs[gate_req_of(a.reqs, a.num_reqs, item)];
        const uint32_t k = item - rq.offset;
        a1 = rq.a + static_cast<size_t>(k) * a.n;
        a2 = a1;
        b = rq.b[k];
    } else {
        const uint32_t in = item / a.levels_tv;
        a1 = a.a1 + static_cast<size_t>(in) * a.n;
        a2 = a.a2 ? a.a2 + static_cast<size_t>(in) * a.n : a1;
        b = gate_b(a.gate, a.b1[in], a.b2 ? a.b2[in] : 0u);
    }
}

// Split-FP32 form of k_gate_blind_rotate on the 32-bit torus (one coefficient per step).  The
// transforms run in FP32.  Each key polynomial k is held as LIMBS FP32 spectra: LIMBS = 2
// splits k = lo + 2^S hi (mod 2^32), S = log2 N + 14 (24 at N = 1024, 25 at N = 2048), into
// its signed S-bit residue lo and the signed (32 - S)-bit hi; LIMBS = 1 keeps the centred k.
// The three digit spectra of a half serve every limb; per limb the partial sums of the own
// column are exchanged between the halves as in the FP64 kernel, inverse-transformed,
// rounded to integers, and the limbs are recombined in 32-bit integers (lo + (hi << S)).
// With digits |d| <= 2^6 the hi limb's sums stay near 2^18 in magnitude, far inside FP32's
// 24-bit mantissa (FP32 error ~0.05 rms against the 0.5 that rounding tolerates), so they
// round to the exact integers and the result differs from the exact product by the FP32
// error of the lo limb alone (about 2^11 rms of the 2^32 torus per external product; about
// 2^19 with LIMBS = 1).  This is the limb split of the reference's split-FFT backend
// (bitwise/src/cirbts/cirbts-init.cu:1084-1140, FP64 limbs recombined with base powers mod
// Q) carried to FP32 on the torus, where only the top limb has to be exact.
template <int LOGN, int LIMBS>
__global__ void __launch_bounds__(GateCfg<LOGN>::T, GateCfg<LOGN>::MIN_BLOCKS)
    k_gate_blind_rotate_f32(const GateArgs a) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, T = 2 * TH, TWO_N = 2 * N;
    constexpr uint32_t SH = 32 - (LOGN + 1);  // torus -> Z_2N
    constexpr uint32_t SPLIT = LOGN + 14;     // lo limb bits
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    float2* fs = reinterpret_cast<float2*>(smem);                   // [2][LIMBS][M]
    float2* tab = fs + 2 * LIMBS * M;                               // FftTab<LOGM> in FP32
    uint32_t* acc = reinterpret_cast<uint32_t*>(tab + Tb::size());  // [2][N] torus values
    uint32_t* dig = acc + 2 * N;                                    // [2][levels][M] packed pairs
    const float2* tws = tab + Tb::twist_off();
    const uint32_t tid = threadIdx.x, h = tid / TH, ht = tid % TH;
    uint32_t* my_acc = acc + h * N;
    float2* my_fs = fs + h * LIMBS * M;
    const uint32_t levels = a.levels, bg = a.bg_bits, l2 = 2 * levels;
    uint32_t off = 1u << (32 - levels * bg - 1);  // rounding of the dropped bits
    for (uint32_t k = 0; k < levels; ++k) off += (1u << (bg - 1)) << (32 - (k + 1) * bg);
    auto half_bar = [h]() {
        if (h == 0) asm volatile("bar.sync 1, %0;" ::"n"(TH) : "memory");
        else asm volatile("bar.sync 2, %0;" ::"n"(TH) : "memory");
    };
    auto ms = [](uint32_t x) { return ((x + (1u << (SH - 1))) >> SH) & (TWO_N - 1); };

    for (uint32_t i = tid; i < Tb::size(); i += T) tab[i] = a.tab32[i];
    for (uint32_t item = blockIdx.x; item < a.items; item += gridDim.x) {
        const uint32_t* a1;
        const uint32_t* a2;
        uint32_t b;
        gate_item_inputs(a, item, a1, a2, b);
        const uint32_t mu = static_cast<uint32_t>(a.mu[item % a.levels_tv]);
        const uint32_t b_add = static_cast<uint32_t>(a.b_add[item % a.levels_tv]);
        {
            const uint32_t bt = ms(b);
            for (uint32_t i = tid; i < N; i += T) {
                acc[i] = 0;
                const uint32_t sp = (i + bt) & (TWO_N - 1);
                const uint32_t tv = a.tv ? __ldg(a.tv + (sp & (N - 1))) : mu;
                acc[N + i] = sp < N ? tv : 0u - tv;
            }
        }
        __syncthreads();

        for (uint32_t step = 0; step < a.n; ++step) {
            const uint32_t at = ms(a.reqs ? __ldg(a1 + step) : gate_a(a.gate, __ldg(a1 + step), __ldg(a2 + step)));
            if (at == 0) continue;  // X^0 - 1 = 0: the step adds nothing (uniform over the CTA)
            for (uint32_t e = ht; e < M; e += TH) {
                const uint32_t wr = my_acc[e] + off, wi = my_acc[e + M] + off;
                uint32_t* dst = dig + h * levels * M + e;
                for (uint32_t k = 0; k < levels; ++k) {
                    const uint32_t s = 32 - (k + 1) * bg, mask = (1u << bg) - 1, half = 1u << (bg - 1);
                    const int32_t dr = static_cast<int32_t>((wr >> s) & mask) - static_cast<int32_t>(half);
                    const int32_t di = static_cast<int32_t>((wi >> s) & mask) - static_cast<int32_t>(half);
                    dst[k * M] = (static_cast<uint32_t>(dr) & 0xffffu) | (static_cast<uint32_t>(di) << 16);
                }
            }
            half_bar();
            const float2* ek = a.bskf32 + static_cast<size_t>(step) * l2 * 2 * LIMBS * M + ht;
            float2 y[2][LIMBS][8];
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int l = 0; l < LIMBS; ++l)
#pragma unroll
                    for (int j = 0; j < 8; ++j) y[c][l][j] = make_float2(0.f, 0.f);
            for (uint32_t d = 0; d < levels; ++d) {
                const uint32_t* dsrc = dig + (h * levels + d) * M;
                float2 x[8];
                fft_forward_to_regs<LOGM>(
                    my_fs, ht, tab,
                    [&](int j, uint32_t e) {
                        const uint32_t v = dsrc[e];
                        const float re = static_cast<float>(static_cast<int16_t>(v & 0xffffu));
                        const float im = static_cast<float>(static_cast<int16_t>(v >> 16));
                        return cmul(make_float2(re, im), gate_twist<LOGM>(tws, j, e));
                    },
                    x, half_bar);
                const float2* kr = ek + static_cast<size_t>(2 * d + h) * 2 * LIMBS * M;  // [column][limb][M]
#pragma unroll
                for (int c = 0; c < 2; ++c)
#pragma unroll
                    for (int l = 0; l < LIMBS; ++l)
#pragma unroll
                        for (int j = 0; j < 8; ++j) cfma(y[c][l][j], x[j], __ldg(kr + (c * LIMBS + l) * M + j * TH));
                half_bar();
            }
            // column 1 - h of every limb goes to the other half, column h stays
#pragma unroll
            for (int l = 0; l < LIMBS; ++l)
#pragma unroll
                for (int j = 0; j < 8; ++j) my_fs[l * M + cswz_of<float2>(8 * ht + j)] = h ? y[0][l][j] : y[1][l][j];
            __syncthreads();
            float2 z[LIMBS][8];
            {
                const float2* take = fs + (1 - h) * LIMBS * M;
#pragma unroll
                for (int l = 0; l < LIMBS; ++l)
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        z[l][j] = cadd(h ? y[1][l][j] : y[0][l][j], take[l * M + cswz_of<float2>(8 * ht + j)]);
            }
            __syncthreads();
            uint32_t tre[8], tim[8];
            constexpr float inv_m = 1.0f / M;
#pragma unroll
            for (int l = 0; l < LIMBS; ++l) {
                fft_inverse_from_regs<LOGM>(
                    my_fs, ht, tab, z[l],
                    [&](int j, uint32_t e, float2 v) {
                        const float2 u = cmulc(v, gate_twist<LOGM>(tws, j, e));
                        const uint32_t re = static_cast<uint32_t>(__float2ll_rn(u.x * inv_m));
                        const uint32_t im = static_cast<uint32_t>(__float2ll_rn(u.y * inv_m));
                        if (l == 0) {
                            tre[j] = re;
                            tim[j] = im;
                        } else {
                            tre[j] += re << SPLIT;
                            tim[j] += im << SPLIT;
                        }
                    },
                    half_bar);
                half_bar();
            }
            uint32_t* tsm = reinterpret_cast<uint32_t*>(my_fs);  // N words (the buffer holds LIMBS * 8 M bytes)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                tsm[ht + j * TH] = tre[j];
                tsm[ht + j * TH + M] = tim[j];
            }
            half_bar();
#pragma unroll 4
            for (uint32_t k = 0; k < N / TH; ++k) {
                const uint32_t i = ht + k * TH;
                const uint32_t s = (i + TWO_N - at) & (TWO_N - 1);
                const uint32_t v = (s < N) ? tsm[s] : 0u - tsm[s - N];
                my_acc[i] += v - tsm[i];
            }
        }
        __syncthreads();
        // sample extract of coefficient 0: a'_0 = a_0, a'_i = -a_(N-i), b' = b_0
        uint32_t* out = reinterpret_cast<uint32_t*>(a.ext) + static_cast<size_t>(item) * (N + 1);
        for (uint32_t i = tid; i <= N; i += T) {
            uint32_t v;
            if (i == N) v = acc[N] + b_add;
            else if (i == 0) v = acc[0];
            else v = 0u - acc[N - i];
            out[i] = v;
        }
        __syncthreads();  // acc is re-initialised by the next item
    }
}

// Grouped (multi-bit) form of k_gate_blind_rotate, the reference's CIRBTS_PBS_MULTIBIT key
// grouping (bitwise/src/cirbts/cirbts-init.cu:376-530, kernel.cu:4585-4771) on the torus: per
// group of MB coefficients acc += sum_S m_S (acc (x) RGSW(prod_{i in S} s_i)), m_S =
// prod_{i in S} (X^{a_i} - 1), with the combined key sum_S m_S(psi) K_S formed per spectrum
// slot (the structure of k_blind_rotate_fft_mb: c_i per slot once per group in shared memory,
// the 16 key spectra of one subset loaded together).  Groups whose rotations are all 0 are
// skipped.  Keys: [groups][2^MB - 1][2*levels][2][M] spectra.
template <int LOGN>
struct GateMbCfg {
    static constexpr uint32_t T = (1u << LOGN) / 8;
    static constexpr int MIN_BLOCKS = LOGN <= 10 ? 2 : 1;  // the whole register file per CTA pair / CTA
};

template <int LOGN, typename TT, int MB>
__global__ void __launch_bounds__(GateMbCfg<LOGN>::T, GateMbCfg<LOGN>::MIN_BLOCKS)
    k_gate_blind_rotate_mb(const GateArgs a) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, T = 2 * TH, TWO_N = 2 * N;
    constexpr uint32_t SH = 32 - (LOGN + 1);  // torus -> Z_2N
    constexpr uint32_t KS = (1u << MB) - 1u;
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    double2* fs = reinterpret_cast<double2*>(smem);             // [2][M]
    double2* tab = fs + 2 * M;                                  // FftTab<LOGM>
    TT* acc = reinterpret_cast<TT*>(tab + Tb::size());         // [2][N] torus values
    uint32_t* dig = reinterpret_cast<uint32_t*>(acc + 2 * N);  // [2][levels][M] packed pairs
    double2* cbuf = reinterpret_cast<double2*>(dig + 2 * a.levels * M);  // [MB][8][T]
    const double2* tws = tab + Tb::twist_off();
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const uint32_t h = tid / TH, ht = tid % TH;
    TT* my_acc = acc + h * N;
    double2* my_fs = fs + h * M;
    const uint32_t levels = a.levels, bg = a.bg_bits;
    constexpr uint32_t W = 8 * sizeof(TT);
    TT off = TT(1) << (W - levels * bg - 1);
    for (uint32_t k = 0; k < levels; ++k) off += (TT(1) << (bg - 1)) << (W - (k + 1) * bg);
    auto half_bar = [h]() {
        if (h == 0) asm volatile("bar.sync 1, %0;" ::"n"(TH) : "memory");
        else asm volatile("bar.sync 2, %0;" ::"n"(TH) : "memory");
    };
    auto ms = [](uint32_t x) { return ((x + (1u << (SH - 1))) >> SH) & (TWO_N - 1); };

    for (uint32_t i = tid; i < Tb::size(); i += T) tab[i] = a.tab[i];
    const uint32_t l2 = 2 * levels;
    const size_t kstride = static_cast<size_t>(l2) * 2 * M;
    const uint32_t groups = (a.n + MB - 1) / MB;
    for (uint32_t item = ct; item < a.items; item += gridDim.x) {
        const uint32_t* a1;
        const uint32_t* a2;
        uint32_t b;
        if (a.reqs) {
            const GateReq& rq = a.reqs[gate_req_of(a.reqs, a.num_reqs, item)];
            const uint32_t k = item - rq.offset;
            a1 = rq.a + static_cast<size_t>(k) * a.n;
            a2 = a1;
            b = rq.b[k];
        } else {
            const uint32_t in = item / a.levels_tv;
            a1 = a.a1 + static_cast<size_t>(in) * a.n;
            a2 = a.a2 ? a.a2 + static_cast<size_t>(in) * a.n : a1;
            b = gate_b(a.gate, a.b1[in], a.b2 ? a.b2[in] : 0u);
        }
        const TT mu = static_cast<TT>(a.mu[item % a.levels_tv]), b_add = static_cast<TT>(a.b_add[item % a.levels_tv]);
        {
            const uint32_t bt = ms(b);
            for (uint32_t i = tid; i < N; i += T) {
                acc[i] = 0;
                const uint32_t sp = (i + bt) & (TWO_N - 1);
                const TT tv = a.tv ? static_cast<TT>(__ldg(a.tv + (sp & (N - 1)))) : mu;
                acc[N + i] = sp < N ? tv : TT(0) - tv;
            }
        }
        __syncthreads();

        for (uint32_t g = 0; g < groups; ++g) {
            uint32_t at[MB];
            uint32_t any = 0;
#pragma unroll
            for (int i = 0; i < MB; ++i) {
                const uint32_t idx = g * MB + i;
                at[i] = idx < a.n ? ms(a.reqs ? __ldg(a1 + idx) : gate_a(a.gate, __ldg(a1 + idx), __ldg(a2 + idx)))
                                  : 0u;
                any |= at[i];
            }
            if (any == 0) continue;  // every m_S is 0 (uniform over the CTA)
#pragma unroll
            for (int i = 0; i < MB; ++i) {
                const double2 ub = zeta_pow<LOGN>(tws, mult_base<LOGN>(ht, at[i]));
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t r3 = ((j & 1) << 2) | (j & 2) | ((j >> 2) & 1);
                    const uint32_t k = (at[i] * r3) & 7u;
                    double2 w = tab[(k & 3u) * (M / 8)];
                    if (k & 4u) w = make_double2(-w.x, -w.y);
                    const double2 v = cmul(ub, w);
                    cbuf[(i * 8 + j) * T + tid] = make_double2(v.x - 1.0, v.y);
                }
            }
            for (uint32_t e = ht; e < M; e += TH) {
                const TT wr = my_acc[e] + off, wi = my_acc[e + M] + off;
                uint32_t* dst = dig + h * levels * M + e;
                for (uint32_t k = 0; k < levels; ++k) {
                    const uint32_t sft = W - (k + 1) * bg, mask = (1u << bg) - 1, half = 1u << (bg - 1);
                    const int32_t dr = static_cast<int32_t>((wr >> sft) & mask) - static_cast<int32_t>(half);
                    const int32_t di = static_cast<int32_t>((wi >> sft) & mask) - static_cast<int32_t>(half);
                    dst[k * M] = (static_cast<uint32_t>(dr) & 0xffffu) | (static_cast<uint32_t>(di) << 16);
                }
            }
            half_bar();
            const double2* gk = a.bskf + static_cast<size_t>(g) * KS * kstride + ht;
            double2 y0[8], y1[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) y0[j] = y1[j] = make_double2(0.0, 0.0);
            for (uint32_t d = 0; d < levels; ++d) {
                const uint32_t* dsrc = dig + (h * levels + d) * M;
                double2 x[8];
                fft_forward_to_regs<LOGM>(
                    my_fs, ht, tab,
                    [&](int j, uint32_t e) {
                        const uint32_t v = dsrc[e];
                        const double re = static_cast<double>(static_cast<int16_t>(v & 0xffffu));
                        const double im = static_cast<double>(static_cast<int16_t>(v >> 16));
                        return cmul(make_double2(re, im), gate_twist<LOGM>(tws, j, e));
                    },
                    x, half_bar);
                const double2* k0 = gk + static_cast<size_t>(2 * d + h) * 2 * M;
                double2 kc0[8], kc1[8];
#pragma unroll
                for (int sub = 0; sub < static_cast<int>(KS); ++sub) {
                    double2 ka[8], kb[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        ka[j] = __ldg(k0 + sub * kstride + j * TH);
                        kb[j] = __ldg(k0 + sub * kstride + M + j * TH);
                    }
                    const uint32_t mask = mb_key_mask(MB, sub);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        double2 m = make_double2(1.0, 0.0);
                        bool first = true;
#pragma unroll
                        for (int i = 0; i < MB; ++i)
                            if (mask & (1u << i)) {
                                const double2 c = cbuf[(i * 8 + j) * T + tid];
                                m = first ? c : cmul(m, c);
                                first = false;
                            }
                        if (sub == 0) {
                            kc0[j] = cmul(m, ka[j]);
                            kc1[j] = cmul(m, kb[j]);
                        } else {
                            cfma(kc0[j], m, ka[j]);
                            cfma(kc1[j], m, kb[j]);
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    cfma(y0[j], x[j], kc0[j]);
                    cfma(y1[j], x[j], kc1[j]);
                }
                half_bar();
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) my_fs[cswz(8 * ht + j)] = h ? y0[j] : y1[j];
            __syncthreads();
            {
                const double2* take = fs + (1 - h) * M;
#pragma unroll
                for (int j = 0; j < 8; ++j) y0[j] = cadd(h ? y1[j] : y0[j], take[cswz(8 * ht + j)]);
            }
            __syncthreads();
            constexpr double inv_m = 1.0 / M;
            // the monomials are in the combined keys: add the rounded product in place
            fft_inverse_from_regs<LOGM>(
                my_fs, ht, tab, y0,
                [&](int j, uint32_t e, double2 v) {
                    const double2 u = cmulc(v, gate_twist<LOGM>(tws, j, e));
                    my_acc[e] += to_torus<TT>(u.x * inv_m);
                    my_acc[e + M] += to_torus<TT>(u.y * inv_m);
                },
                half_bar);
        }
        __syncthreads();
        TT* out = reinterpret_cast<TT*>(a.ext) + static_cast<size_t>(item) * (N + 1);
        for (uint32_t i = tid; i <= N; i += T) {
            TT v;
            if (i == N) v = acc[N] + b_add;
            else if (i == 0) v = acc[0];
            else v = TT(0) - acc[N - i];
            out[i] = v;
        }
        __syncthreads();
    }
}

// LWE key switch N -> n of one extracted ciphertext per blockIdx.y; thread j < n + 1 of the
// grid owns output coefficient j (j = n is b).  The digits of a'_i are the same for every
// thread, so the inner loop is uniform and each step reads one coalesced key row segment.
__global__ void __launch_bounds__(256) k_gate_keyswitch(const uint32_t* __restrict__ ext,
                                                        const uint32_t* __restrict__ ksk, uint32_t n, uint32_t N,
                                                        uint32_t ks_bits, uint32_t ks_levels,
                                                        uint32_t* __restrict__ out_a, uint32_t* __restrict__ out_b,
                                                        const GateReq* __restrict__ reqs, uint32_t num_reqs) {
    extern __shared__ uint32_t s_ext[];
    const uint32_t ct = blockIdx.x;  // item
    const uint32_t* src = ext + static_cast<size_t>(ct) * (N + 1);
    for (uint32_t i = threadIdx.x; i <= N; i += blockDim.x) s_ext[i] = src[i];
    __syncthreads();
    const uint32_t j = blockIdx.y * blockDim.x + threadIdx.x;
    if (j > n) return;
    const uint32_t base = 1u << ks_bits, round = 1u << (32 - ks_levels * ks_bits - 1);
    uint32_t accv = (j == n) ? s_ext[N] : 0u;
    for (uint32_t i = 0; i < N; ++i) {
        const uint32_t x = s_ext[i] + round;
        const uint32_t* rows = ksk + static_cast<size_t>(i) * ks_levels * (base - 1) * (n + 1) + j;
        for (uint32_t l = 0; l < ks_levels; ++l) {
            const uint32_t v = (x >> (32 - (l + 1) * ks_bits)) & (base - 1);
            if (v) accv -= __ldg(rows + (static_cast<size_t>(l) * (base - 1) + (v - 1)) * (n + 1));
        }
    }
    uint32_t* oa = out_a;
    uint32_t* ob = out_b;
    uint32_t k = ct;
    if (reqs) {
        const GateReq& rq = reqs[gate_req_of(reqs, num_reqs, ct)];
        oa = rq.out_a;
        ob = rq.out_b;
        k = ct - rq.offset;
    }
    if (j < n) oa[static_cast<size_t>(k) * n + j] = accv;
    else ob[k] = accv;
}

template <int LOGN, typename TT>
static cudaError_t gate_br_launch(const GateArgs& a, uint32_t grid, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    const size_t smem = (2ull * M + FftTab<LOGN - 1>::size()) * sizeof(double2) + 2ull * N * sizeof(TT) +
                        2ull * a.levels * M * sizeof(uint32_t);
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_gate_blind_rotate<LOGN, TT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_gate_blind_rotate<LOGN, TT><<<grid, GateCfg<LOGN>::T, smem, s>>>(a);
    return cudaGetLastError();
}

template <int LOGN, typename TT, int MB>
static cudaError_t gate_br_mb_launch(const GateArgs& a, uint32_t grid, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    const size_t smem = (2ull * M + FftTab<LOGN - 1>::size()) * sizeof(double2) + 2ull * N * sizeof(TT) +
                        2ull * a.levels * M * sizeof(uint32_t) + MB * 8ull * GateMbCfg<LOGN>::T * sizeof(double2);
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_gate_blind_rotate_mb<LOGN, TT, MB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_gate_blind_rotate_mb<LOGN, TT, MB><<<grid, GateMbCfg<LOGN>::T, smem, s>>>(a);
    return cudaGetLastError();
}

template <int LOGN, int LIMBS>
static cudaError_t gate_br_f32_launch(const GateArgs& a, uint32_t grid, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    const size_t smem = (2ull * LIMBS * M + FftTab<LOGN - 1>::size()) * sizeof(float2) + 2ull * N * sizeof(uint32_t) +
                        2ull * a.levels * M * sizeof(uint32_t);
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_gate_blind_rotate_f32<LOGN, LIMBS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_gate_blind_rotate_f32<LOGN, LIMBS><<<grid, GateCfg<LOGN>::T, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename TT>
static cudaError_t gate_br_dispatch(const GateArgs& a, uint32_t N, uint32_t grid, cudaStream_t s) {
    if (a.fft_mode != 0) {  // FP32 external products: 32-bit torus, one coefficient per step
        if constexpr (std::is_same<TT, uint32_t>::value) {
            if (a.mb > 1 || !a.bskf32 || !a.tab32) return cudaErrorInvalidValue;
            if (a.fft_mode == 1) {
                if (N == 1024) return gate_br_f32_launch<10, 2>(a, grid, s);
                if (N == 2048) return gate_br_f32_launch<11, 2>(a, grid, s);
            } else if (a.fft_mode == 2) {
                if (N == 1024) return gate_br_f32_launch<10, 1>(a, grid, s);
                if (N == 2048) return gate_br_f32_launch<11, 1>(a, grid, s);
            }
        }
        return cudaErrorInvalidValue;
    }
    if (a.mb <= 1) {
        if (N == 1024) return gate_br_launch<10, TT>(a, grid, s);
        if (N == 2048) return gate_br_launch<11, TT>(a, grid, s);
        return cudaErrorInvalidValue;
    }
    if (a.mb == 2) {
        if (N == 1024) return gate_br_mb_launch<10, TT, 2>(a, grid, s);
        if (N == 2048) return gate_br_mb_launch<11, TT, 2>(a, grid, s);
    } else if (a.mb == 3) {
        if (N == 1024) return gate_br_mb_launch<10, TT, 3>(a, grid, s);
        if (N == 2048) return gate_br_mb_launch<11, TT, 3>(a, grid, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t gate_blind_rotate(const GateArgs& a, uint32_t N, uint32_t grid, cudaStream_t s) {
    return gate_br_dispatch<uint32_t>(a, N, grid, s);
}

cudaError_t gate_blind_rotate64(const GateArgs& a, uint32_t N, uint32_t grid, cudaStream_t s) {
    return gate_br_dispatch<uint64_t>(a, N, grid, s);
}

// host helpers shared with the torus circuit bootstrap
uint32_t torus_from_double(double x) {  // x in torus units (any real), rounded to 2^-32
    const double f = x - std::floor(x);
    return static_cast<uint32_t>(static_cast<uint64_t>(std::llround(f * 4294967296.0)));
}

uint32_t torus_noise(Rng& rng, double sigma) {
    return static_cast<uint32_t>(static_cast<int64_t>(std::llround(rng.gaussian() * sigma * 4294967296.0)));
}

// b += a * z (negacyclic, z binary), mod 2^32
void mul_binary_acc(const uint32_t* a, const int32_t* z, uint32_t N, uint32_t* b) {
    for (uint32_t j = 0; j < N; ++j) {
        if (!z[j]) continue;
        for (uint32_t i = 0; i < N; ++i) {
            if (i + j < N) b[i + j] += a[i];
            else b[i + j - N] -= a[i];
        }
    }
}

using cld = std::complex<long double>;

// tables of the host transform: w[e] = exp(2 pi i e / M) (e < M/2), twist[e] = exp(i pi e / N)
template <int LOGM>
static void host_fft_tables_ld(std::vector<cld>& w, std::vector<cld>& twist) {
    constexpr uint32_t M = 1u << LOGM, N = 2 * M;
    const long double pi = 3.141592653589793238462643383279502884L;
    w.resize(M / 2);
    twist.resize(M);
    for (uint32_t e = 0; e < M / 2; ++e) w[e] = std::polar(1.0L, 2.0L * pi * e / M);
    for (uint32_t e = 0; e < M; ++e) twist[e] = std::polar(1.0L, pi * e / N);
}

// folded transform of one real polynomial given by coef(e), e < N: zz[e] = (c_e + i c_(e+M))
// zeta^e, then decimation in frequency (natural order in, bit-reversed out, the order of
// fft_core.cuh's spectra before their slot-major placement (e % 8) * (M / 8) + e / 8)
template <int LOGM, class Coef>
static void host_fold_fft_ld(Coef coef, const std::vector<cld>& w, const std::vector<cld>& twist,
                             std::vector<cld>& zz) {
    constexpr uint32_t M = 1u << LOGM;
    zz.resize(M);
    for (uint32_t e = 0; e < M; ++e) zz[e] = cld(coef(e), coef(e + M)) * twist[e];
    for (size_t hh = M / 2; hh >= 1; hh /= 2) {
        const size_t stride = M / (2 * hh);
        for (size_t s0 = 0; s0 < M; s0 += 2 * hh)
            for (size_t j = 0; j < hh; ++j) {
                const cld u = zz[s0 + j], v = zz[s0 + j + hh];
                zz[s0 + j] = u + v;
                zz[s0 + j + hh] = (u - v) * w[j * stride];
            }
        if (hh == 1) break;
    }
}

template <class F>
static void host_parallel_for(size_t count, F f) {
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th)
        pool.emplace_back([&, th] {
            for (size_t k = th; k < count; k += nth) f(k);
        });
    for (auto& t : pool) t.join();
}

template <int LOGM, typename KT>
static void torus_keys_to_fft_t(const KT* keys, size_t count, std::vector<double2>& out) {
    constexpr uint32_t M = 1u << LOGM, N = 2 * M;
    std::vector<cld> w, twist;
    host_fft_tables_ld<LOGM>(w, twist);
    out.assign(count * M, make_double2(0, 0));
    using ST = typename std::make_signed<KT>::type;  // centred representative
    host_parallel_for(count, [&](size_t k) {
        thread_local std::vector<cld> zz;
        const KT* c = keys + k * N;
        host_fold_fft_ld<LOGM>([c](uint32_t e) { return static_cast<long double>(static_cast<ST>(c[e])); }, w, twist,
                               zz);
        for (uint32_t e = 0; e < M; ++e)
            out[k * M + (e % 8) * (M / 8) + e / 8] =
                make_double2(static_cast<double>(zz[e].real()), static_cast<double>(zz[e].imag()));
    });
}

template <int LOGM>
static void torus_keys_to_fft32_t(const uint32_t* keys, size_t count, uint32_t limbs, std::vector<float2>& out) {
    constexpr uint32_t M = 1u << LOGM, N = 2 * M;
    std::vector<cld> w, twist;
    host_fft_tables_ld<LOGM>(w, twist);
    out.assign(count * limbs * M, make_float2(0, 0));
    constexpr uint32_t split = LOGM + 15;  // lo limb bits, log2 N + 14 (k_gate_blind_rotate_f32)
    host_parallel_for(count * limbs, [&](size_t kl) {
        thread_local std::vector<cld> zz;
        const uint32_t* c = keys + (kl / limbs) * N;
        const uint32_t l = static_cast<uint32_t>(kl % limbs);
        auto coef = [c, l, limbs](uint32_t e) -> long double {
            if (limbs == 1) return static_cast<long double>(static_cast<int32_t>(c[e]));
            const int32_t lo = static_cast<int32_t>(c[e] << (32 - split)) >> (32 - split);  // signed residue
            if (l == 0) return static_cast<long double>(lo);
            return static_cast<long double>(static_cast<int32_t>(c[e] - static_cast<uint32_t>(lo)) >> split);
        };
        host_fold_fft_ld<LOGM>(coef, w, twist, zz);
        for (uint32_t e = 0; e < M; ++e)
            out[kl * M + (e % 8) * (M / 8) + e / 8] =
                make_float2(static_cast<float>(zz[e].real()), static_cast<float>(zz[e].imag()));
    });
}

void torus_keys_to_fft32(uint32_t N, const uint32_t* keys, size_t count, uint32_t limbs, std::vector<float2>& out) {
    if (N == 1024) torus_keys_to_fft32_t<9>(keys, count, limbs, out);
    else if (N == 2048) torus_keys_to_fft32_t<10>(keys, count, limbs, out);
    else out.clear();
}

void torus_keys_to_fft(uint32_t N, const uint32_t* keys, size_t count, std::vector<double2>& out) {
    if (N == 1024) torus_keys_to_fft_t<9>(keys, count, out);
    else if (N == 2048) torus_keys_to_fft_t<10>(keys, count, out);
    else out.clear();
}

void torus_keys_to_fft(uint32_t N, const uint64_t* keys, size_t count, std::vector<double2>& out) {
    if (N == 1024) torus_keys_to_fft_t<9>(keys, count, out);
    else if (N == 2048) torus_keys_to_fft_t<10>(keys, count, out);
    else out.clear();
}

cudaError_t gate_keyswitch(const GateArgs& a, const uint32_t* ksk, uint32_t n, uint32_t N, uint32_t ks_bits,
                           uint32_t ks_levels, uint32_t* out_a, uint32_t* out_b, cudaStream_t s) {
    const dim3 grid(a.items, (n + 1 + 255) / 256);
    k_gate_keyswitch<<<grid, 256, (N + 1) * sizeof(uint32_t), s>>>(static_cast<const uint32_t*>(a.ext), ksk, n, N,
                                                                   ks_bits, ks_levels, out_a, out_b,
                                                                   a.reqs, a.num_reqs);
    return cudaGetLastError();
}

}  // namespace cbs

// ---------------------------------------------------------------------------------------
// host side: keys and the C ABI
// ---------------------------------------------------------------------------------------

using cbs::DevBuf;

#include "gate_context.cuh"

namespace cbs {

cbs_status gate_fill_keys(const cbs_gate_context* ctx, GateArgs& a) {
    if (ctx->br_mb > 1 && !ctx->mb_ready) {
        set_error("gate: grouped keys are not prepared");
        return CBS_ERR_NOT_READY;
    }
    if (ctx->fft_mode != CBS_FFT_FP64 && !ctx->f32_ready) {
        set_error("gate: FP32 key spectra are not prepared");
        return CBS_ERR_NOT_READY;
    }
    a.bskf = ctx->br_mb > 1 ? ctx->d_bskf_mb.p : ctx->d_bskf.p;
    a.mb = ctx->br_mb;
    a.tab = ctx->d_tab.p;
    a.fft_mode = ctx->fft_mode;
    a.bskf32 = ctx->d_bskf32.p;
    a.tab32 = ctx->d_tab32.p;
    return CBS_OK;
}

}  // namespace cbs

namespace {

using cbs::mul_binary_acc;
using cbs::set_error;
using cbs::torus_noise;

cbs_status validate_gate(const cbs_gate_params& p) {
    CBS_CHECK_ARG(p.N == 1024 || p.N == 2048, "gate: N must be 1024 or 2048");
    CBS_CHECK_ARG(p.n >= 1 && p.n <= 4096, "gate: n out of range");
    CBS_CHECK_ARG(p.bg_bits >= 1 && p.bg_bits <= 15 && p.levels >= 1 && p.levels <= 4 && p.bg_bits * p.levels <= 30,
                  "gate: need bg_bits <= 15, levels <= 4, bg_bits * levels <= 30");
    CBS_CHECK_ARG(p.ks_base_bits >= 1 && p.ks_base_bits <= 8 && p.ks_levels >= 1 &&
                      p.ks_base_bits * p.ks_levels <= 31,
                  "gate: key-switch base and levels out of range");
    CBS_CHECK_ARG(p.sigma_lwe >= 0 && p.sigma_rlwe >= 0 && p.sigma_lwe < 0.01 && p.sigma_rlwe < 0.01,
                  "gate: noise out of range");
    // 2^(bg-1) * 2^31 * N * 2*levels must stay below 2^52 for the FFT products to round exactly
    const double bound = std::ldexp(1.0, static_cast<int>(p.bg_bits) - 1 + 31) * p.N * 2 * p.levels;
    CBS_CHECK_ARG(bound < std::ldexp(1.0, 52), "gate: parameters exceed the exact FP64 product range");
    return CBS_OK;
}

}  // namespace

extern "C" {

cbs_status cbs_gate_params_default(cbs_gate_params* out) {
    CBS_CHECK_ARG(out, "gate_params_default: null argument");
    out->n = 636;
    out->N = 1024;
    out->bg_bits = 7;
    out->levels = 3;
    out->ks_base_bits = 2;
    out->ks_levels = 8;
    out->sigma_lwe = std::ldexp(1.0, -15);
    out->sigma_rlwe = std::ldexp(1.0, -25);
    return CBS_OK;
}

cbs_status cbs_gate_context_create(const cbs_gate_params* params, uint32_t max_batch, cbs_gate_context** out) {
    CBS_CHECK_ARG(params && out, "gate_context_create: null argument");
    *out = nullptr;
    CBS_CHECK_ARG(max_batch >= 1 && max_batch <= (1u << 22), "gate_context_create: max_batch out of range");
    if (cbs_status st = validate_gate(*params)) return st;
    auto* c = new (std::nothrow) cbs_gate_context();
    if (!c) {
        set_error("gate_context_create: host allocation failed");
        return CBS_ERR_OOM;
    }
    std::unique_ptr<cbs_gate_context> guard(c);
    c->p = *params;
    c->max_batch = max_batch;
    CBS_CUDA_TRY(c->d_ext.alloc(static_cast<size_t>(max_batch) * (params->N + 1)));
    CBS_CUDA_TRY(c->d_tmp_a.alloc(static_cast<size_t>(max_batch) * params->n));
    CBS_CUDA_TRY(c->d_tmp_b.alloc(max_batch));
    *out = guard.release();
    return CBS_OK;
}

cbs_status cbs_gate_context_destroy(cbs_gate_context* ctx) {
    delete ctx;
    return CBS_OK;
}

}  // extern "C"

namespace {

// seeded host key generation (no device): s (n), z (N) binary; BSK rows 2k+c = RLWE_z(0) with
// s_i * 2^(32-(k+1)*bg_bits) added to component c; KSK rows LWE_s(v * z_i * 2^(32-(l+1)*ks_bits))
void gate_keys_host(const cbs_gate_params& p, uint64_t seed, std::vector<int32_t>& s_out, std::vector<int32_t>& z_out,
                    std::vector<uint32_t>& bsk, std::vector<uint32_t>& ksk) {
    const uint32_t n = p.n, N = p.N, L = p.levels, base = 1u << p.ks_base_bits;
    cbs::Rng rng(seed ^ 0x6a7e5b07c0ffee11ull);
    s_out.assign(n, 0);
    z_out.assign(N, 0);
    for (auto& v : s_out) v = static_cast<int32_t>(rng.uniform(2));
    for (auto& v : z_out) v = static_cast<int32_t>(rng.uniform(2));
    bsk.assign(static_cast<size_t>(n) * 2 * L * 2 * N, 0);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t r = 0; r < 2 * L; ++r) {
            uint32_t* ra = bsk.data() + ((static_cast<size_t>(i) * 2 * L + r) * 2) * N;
            uint32_t* rb = ra + N;
            for (uint32_t e = 0; e < N; ++e) {
                ra[e] = static_cast<uint32_t>(rng.next());
                rb[e] = torus_noise(rng, p.sigma_rlwe);
            }
        }
    {  // b += a * z for every row, in parallel (binary z: shifted additions)
        const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        const size_t rows = static_cast<size_t>(n) * 2 * L;
        for (unsigned th = 0; th < nth; ++th)
            pool.emplace_back([&, th] {
                for (size_t r = th; r < rows; r += nth) {
                    uint32_t* ra = bsk.data() + r * 2 * N;
                    mul_binary_acc(ra, z_out.data(), N, ra + N);
                }
            });
        for (auto& t : pool) t.join();
    }
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t k = 0; k < L; ++k)
            for (uint32_t c = 0; c < 2; ++c) {
                uint32_t* row = bsk.data() + ((static_cast<size_t>(i) * 2 * L + 2 * k + c) * 2 + c) * N;
                row[0] += static_cast<uint32_t>(s_out[i]) << (32 - (k + 1) * p.bg_bits);
            }
    ksk.assign(static_cast<size_t>(N) * p.ks_levels * (base - 1) * (n + 1), 0);
    for (uint32_t i = 0; i < N; ++i)
        for (uint32_t l = 0; l < p.ks_levels; ++l)
            for (uint32_t v = 1; v < base; ++v) {
                uint32_t* row =
                    ksk.data() + ((static_cast<size_t>(i) * p.ks_levels + l) * (base - 1) + v - 1) * (n + 1);
                uint32_t b = torus_noise(rng, p.sigma_lwe);
                for (uint32_t j = 0; j < n; ++j) {
                    row[j] = static_cast<uint32_t>(rng.next());
                    if (s_out[j]) b += row[j];
                }
                b += (v * static_cast<uint32_t>(z_out[i])) << (32 - (l + 1) * p.ks_base_bits);
                row[n] = b;
            }
}

// Grouped keys RGSW_z(prod_{i in S} s_i) for every non-empty subset S of each group of mb
// LWE coefficients (rows 2k + c add the product times 2^(32 - (k+1) bg) to component c), one
// generator per row so the keys do not depend on the thread count.
void gate_mb_keys_host(const cbs_gate_params& p, const std::vector<int32_t>& s, const std::vector<int32_t>& z,
                       uint32_t mb, uint64_t seed, std::vector<uint32_t>& out) {
    const uint32_t n = p.n, N = p.N, L = p.levels, K = cbs::mb_subsets(mb), groups = (n + mb - 1) / mb;
    const size_t rows = static_cast<size_t>(groups) * K * 2 * L;
    out.assign(rows * 2 * N, 0);
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th)
        pool.emplace_back([&, th] {
            for (size_t r = th; r < rows; r += nth) {
                cbs::Rng rr(seed ^ (0x9e3779b97f4a7c15ull * (r + 1)));
                uint32_t* ra = out.data() + r * 2 * N;
                uint32_t* rb = ra + N;
                for (uint32_t e = 0; e < N; ++e) {
                    ra[e] = static_cast<uint32_t>(rr.next());
                    rb[e] = torus_noise(rr, p.sigma_rlwe);
                }
                mul_binary_acc(ra, z.data(), N, rb);
                const uint32_t g = static_cast<uint32_t>(r / (K * 2 * L));
                const uint32_t kk = static_cast<uint32_t>((r / (2 * L)) % K), row = static_cast<uint32_t>(r % (2 * L));
                const uint32_t mask = cbs::mb_subset_mask(mb, kk);
                uint32_t prod = 1;
                for (uint32_t i = 0; i < mb; ++i)
                    if (mask & (1u << i)) prod &= (g * mb + i < n) ? static_cast<uint32_t>(s[g * mb + i]) : 0u;
                (row % 2 ? rb : ra)[0] += prod << (32 - (row / 2 + 1) * p.bg_bits);
            }
        });
    for (auto& t : pool) t.join();
}

constexpr uint64_t kGateMbSeedTweak = 0x67617465206d6275ull;

// FP32 key-limb spectra of the one-bit keys and the FP32 copy of the transform table
cbs_status gate_prepare_f32(cbs_gate_context* ctx) {
    if (ctx->fft_mode == CBS_FFT_FP64 || ctx->f32_ready || !ctx->keys_ready) return CBS_OK;
    const uint32_t limbs = ctx->fft_mode == CBS_FFT_FP32_SPLIT ? 2 : 1;
    std::vector<float2> spec, tab32;
    std::vector<double2> tab;
    try {
        cbs::torus_keys_to_fft32(ctx->p.N, ctx->bsk.data(), ctx->bsk.size() / ctx->p.N, limbs, spec);
        cbs::fft_tables_host(ctx->p.N, tab);
        tab32.resize(tab.size());
        for (size_t i = 0; i < tab.size(); ++i)
            tab32[i] = make_float2(static_cast<float>(tab[i].x), static_cast<float>(tab[i].y));
    } catch (const std::exception& e) {
        set_error(std::string("gate FP32 keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    CBS_CUDA_TRY(ctx->d_bskf32.upload(spec.data(), spec.size(), nullptr));
    CBS_CUDA_TRY(ctx->d_tab32.upload(tab32.data(), tab32.size(), nullptr));
    CBS_CUDA_TRY(cudaStreamSynchronize(nullptr));
    ctx->f32_ready = true;
    return CBS_OK;
}

// the arithmetic fields of the launch arguments; CBS_ERR_NOT_READY when the selected keys are
// not prepared

cbs_status gate_prepare_mb(cbs_gate_context* ctx) {
    if (ctx->br_mb <= 1 || ctx->mb_ready || !ctx->keys_ready) return CBS_OK;
    std::vector<double2> spec;
    try {
        gate_mb_keys_host(ctx->p, ctx->s, ctx->z, ctx->br_mb, ctx->key_seed ^ kGateMbSeedTweak, ctx->mbk);
        cbs::torus_keys_to_fft(ctx->p.N, ctx->mbk.data(), ctx->mbk.size() / ctx->p.N, spec);
    } catch (const std::exception& e) {
        set_error(std::string("gate multi-bit keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    CBS_CUDA_TRY(ctx->d_bskf_mb.upload(spec.data(), spec.size(), nullptr));
    CBS_CUDA_TRY(cudaStreamSynchronize(nullptr));
    ctx->mb_ready = true;
    return CBS_OK;
}

}  // namespace

extern "C" {

cbs_status cbs_gate_set_multibit(cbs_gate_context* ctx, uint32_t mb) {
    CBS_CHECK_ARG(ctx, "gate_set_multibit: null context");
    CBS_CHECK_ARG(mb >= 1 && mb <= 3, "gate_set_multibit: mb must be 1, 2 or 3");
    CBS_CHECK_ARG(mb == 1 || ctx->fft_mode == CBS_FFT_FP64,
                  "gate_set_multibit: the FP32 external products run one coefficient per step (mb = 1)");
    if (mb != ctx->br_mb) {
        ctx->br_mb = mb;
        ctx->mb_ready = false;
        ctx->mbk.clear();
        ctx->d_bskf_mb.reset();
    }
    return gate_prepare_mb(ctx);
}

cbs_status cbs_gate_set_fft_mode(cbs_gate_context* ctx, uint32_t mode) {
    CBS_CHECK_ARG(ctx, "gate_set_fft_mode: null context");
    CBS_CHECK_ARG(mode == CBS_FFT_FP64 || mode == CBS_FFT_FP32_SPLIT || mode == CBS_FFT_FP32,
                  "gate_set_fft_mode: mode must be CBS_FFT_FP64, CBS_FFT_FP32_SPLIT or CBS_FFT_FP32");
    CBS_CHECK_ARG(mode == CBS_FFT_FP64 || ctx->br_mb <= 1,
                  "gate_set_fft_mode: the FP32 external products run one coefficient per step (mb = 1)");
    // the split's top limb times a digit, summed over N terms, must stay far inside the 24-bit
    // FP32 mantissa for its rounding to be exact: digits of at most 7 bits
    CBS_CHECK_ARG(mode != CBS_FFT_FP32_SPLIT || ctx->p.bg_bits <= 7,
                  "gate_set_fft_mode: split FP32 needs bg_bits <= 7");
    if (mode != ctx->fft_mode) {
        ctx->fft_mode = mode;
        ctx->f32_ready = false;
        ctx->d_bskf32.reset();
        ctx->d_tab32.reset();
    }
    return gate_prepare_f32(ctx);
}

cbs_status cbs_gate_export_mb_bsk(const cbs_gate_context* ctx, uint32_t* out, size_t* words) {
    CBS_CHECK_ARG(ctx && words, "gate_export_mb_bsk: null argument");
    if (ctx->br_mb <= 1 || !ctx->mb_ready) {
        set_error("gate_export_mb_bsk: no grouped keys (select mb > 1 after cbs_gate_keygen)");
        return CBS_ERR_NOT_READY;
    }
    *words = ctx->mbk.size();
    if (out) std::copy(ctx->mbk.begin(), ctx->mbk.end(), out);
    return CBS_OK;
}

cbs_status cbs_gate_generate_keys_host(const cbs_gate_params* params, uint64_t seed, int32_t* s_lwe, int32_t* z_rlwe,
                                       uint32_t* bsk, uint32_t* ksk) {
    CBS_CHECK_ARG(params, "gate_generate_keys_host: null params");
    if (cbs_status st = validate_gate(*params)) return st;
    std::vector<int32_t> s, z;
    std::vector<uint32_t> b, k;
    gate_keys_host(*params, seed, s, z, b, k);
    if (s_lwe) std::copy(s.begin(), s.end(), s_lwe);
    if (z_rlwe) std::copy(z.begin(), z.end(), z_rlwe);
    if (bsk) std::copy(b.begin(), b.end(), bsk);
    if (ksk) std::copy(k.begin(), k.end(), ksk);
    return CBS_OK;
}

cbs_status cbs_gate_keygen(cbs_gate_context* ctx, uint64_t seed) {
    CBS_CHECK_ARG(ctx, "gate_keygen: null context");
    const cbs_gate_params& p = ctx->p;
    const uint32_t N = p.N;
    gate_keys_host(p, seed, ctx->s, ctx->z, ctx->bsk, ctx->ksk);
    std::vector<double2> bskf, tab;
    if (N == 1024) {
        cbs::torus_keys_to_fft(N, ctx->bsk.data(), ctx->bsk.size() / N, bskf);
        cbs::fft_tables_host(N, tab);
    } else {
        cbs::torus_keys_to_fft(N, ctx->bsk.data(), ctx->bsk.size() / N, bskf);
        cbs::fft_tables_host(N, tab);
    }
    CBS_CUDA_TRY(ctx->d_bskf.upload(bskf.data(), bskf.size(), nullptr));
    CBS_CUDA_TRY(ctx->d_tab.upload(tab.data(), tab.size(), nullptr));
    CBS_CUDA_TRY(ctx->d_ksk.upload(ctx->ksk.data(), ctx->ksk.size(), nullptr));
    CBS_CUDA_TRY(cudaStreamSynchronize(nullptr));
    ctx->keys_ready = true;
    ctx->key_seed = seed;
    ctx->mb_ready = false;
    ctx->f32_ready = false;
    if (cbs_status st = gate_prepare_f32(ctx)) return st;
    return gate_prepare_mb(ctx);
}

cbs_status cbs_gate_export_keys(const cbs_gate_context* ctx, int32_t* s_lwe, int32_t* z_rlwe, uint32_t* bsk,
                                uint32_t* ksk) {
    CBS_CHECK_ARG(ctx, "gate_export_keys: null context");
    if (!ctx->keys_ready) {
        set_error("gate_export_keys: no keys (call cbs_gate_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    if (s_lwe) std::copy(ctx->s.begin(), ctx->s.end(), s_lwe);
    if (z_rlwe) std::copy(ctx->z.begin(), ctx->z.end(), z_rlwe);
    if (bsk) std::copy(ctx->bsk.begin(), ctx->bsk.end(), bsk);
    if (ksk) std::copy(ctx->ksk.begin(), ctx->ksk.end(), ksk);
    return CBS_OK;
}

cbs_status cbs_gate_encrypt_bits(const cbs_gate_context* ctx, const uint8_t* h_bits, uint32_t count, uint64_t seed,
                                 uint32_t* h_a, uint32_t* h_b) {
    CBS_CHECK_ARG(ctx && h_bits && h_a && h_b, "gate_encrypt_bits: null argument");
    if (!ctx->keys_ready) {
        set_error("gate_encrypt_bits: no keys (call cbs_gate_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    cbs::Rng rng(seed);
    const uint32_t n = ctx->p.n;
    for (uint32_t k = 0; k < count; ++k) {
        uint32_t b = (h_bits[k] ? (1u << 29) : (0u - (1u << 29))) + torus_noise(rng, ctx->p.sigma_lwe);
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t a = static_cast<uint32_t>(rng.next());
            h_a[static_cast<size_t>(k) * n + j] = a;
            if (ctx->s[j]) b += a;
        }
        h_b[k] = b;
    }
    return CBS_OK;
}

cbs_status cbs_gate_decrypt_bits(const cbs_gate_context* ctx, const uint32_t* h_a, const uint32_t* h_b,
                                 uint32_t count, uint8_t* h_bits) {
    CBS_CHECK_ARG(ctx && h_a && h_b && h_bits, "gate_decrypt_bits: null argument");
    if (!ctx->keys_ready) {
        set_error("gate_decrypt_bits: no keys (call cbs_gate_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    const uint32_t n = ctx->p.n;
    for (uint32_t k = 0; k < count; ++k) {
        uint32_t ph = h_b[k];
        for (uint32_t j = 0; j < n; ++j)
            if (ctx->s[j]) ph -= h_a[static_cast<size_t>(k) * n + j];
        h_bits[k] = static_cast<int32_t>(ph) > 0 ? 1 : 0;
    }
    return CBS_OK;
}

static cbs_status gate_run(cbs_gate_context* ctx, int gate, const uint32_t* d_a1, const uint32_t* d_b1,
                           const uint32_t* d_a2, const uint32_t* d_b2, uint32_t count, uint32_t* d_ext,
                           uint32_t* d_out_a, uint32_t* d_out_b, cudaStream_t s) {
    if (!ctx->keys_ready) {
        set_error("gate: no keys (call cbs_gate_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    if (count == 0) return CBS_OK;
    if (count > ctx->max_batch) {
        set_error("gate: count above the context's max_batch");
        return CBS_ERR_SHAPE_MISMATCH;
    }
    const cbs_gate_params& p = ctx->p;
    cbs::GateArgs a{};
    if (cbs_status st = gate_fill_keys(ctx, a)) return st;
    a.gate = gate;
    a.a1 = d_a1;
    a.b1 = d_b1;
    a.a2 = d_a2;
    a.b2 = d_b2;
    a.n = p.n;
    a.levels = p.levels;
    a.bg_bits = p.bg_bits;
    a.ext = d_ext ? d_ext : ctx->d_ext.p;
    a.items = count;
    a.levels_tv = 1;
    a.mu[0] = 1u << 29;
    CBS_CUDA_TRY(cbs::gate_blind_rotate(a, p.N, count, s));
    if (d_out_a && d_out_b) {
        const dim3 grid(count, (p.n + 1 + 255) / 256);
        cbs::k_gate_keyswitch<<<grid, 256, (p.N + 1) * sizeof(uint32_t), s>>>(
            static_cast<const uint32_t*>(a.ext), ctx->d_ksk.p, p.n, p.N, p.ks_base_bits, p.ks_levels, d_out_a, d_out_b,
            nullptr, 0);
        CBS_LAUNCH_CHECK();
    }
    return CBS_OK;
}

cbs_status cbs_gate_eval_batch_device(cbs_gate_context* ctx, int gate, const uint32_t* d_a1, const uint32_t* d_b1,
                                      const uint32_t* d_a2, const uint32_t* d_b2, uint32_t count, uint32_t* d_out_a,
                                      uint32_t* d_out_b, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && d_a1 && d_b1 && d_a2 && d_b2 && d_out_a && d_out_b, "gate_eval_batch: null argument");
    CBS_CHECK_ARG(gate >= CBS_GATE_OR && gate <= CBS_GATE_XNOR, "gate_eval_batch: unknown gate");
    return gate_run(ctx, gate, d_a1, d_b1, d_a2, d_b2, count, nullptr, d_out_a, d_out_b, stream);
}

cbs_status cbs_gate_bootstrap_batch_device(cbs_gate_context* ctx, const uint32_t* d_a, const uint32_t* d_b,
                                           uint32_t count, uint32_t* d_ext, uint32_t* d_out_a, uint32_t* d_out_b,
                                           cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && d_a && d_b, "gate_bootstrap_batch: null argument");
    CBS_CHECK_ARG((d_out_a == nullptr) == (d_out_b == nullptr), "gate_bootstrap_batch: give both outputs or neither");
    CBS_CHECK_ARG(d_ext || d_out_a, "gate_bootstrap_batch: no output requested");
    return gate_run(ctx, -1, d_a, d_b, nullptr, nullptr, count, d_ext, d_out_a, d_out_b, stream);
}

cbs_status cbs_gate_ragged_plan(cbs_gate_context* ctx, const cbs_gate_request* h_reqs, uint32_t num_reqs,
                                uint32_t grid_ctas) {
    CBS_CHECK_ARG(ctx && (h_reqs || num_reqs == 0), "gate_ragged_plan: null argument");
    if (!ctx->keys_ready) {
        set_error("gate_ragged_plan: no keys (call cbs_gate_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    std::vector<cbs::GateReq> reqs;
    uint64_t items = 0;
    for (uint32_t r = 0; r < num_reqs; ++r) {
        const cbs_gate_request& q = h_reqs[r];
        if (q.count == 0) continue;
        CBS_CHECK_ARG(q.d_a && q.d_b && q.d_out_a && q.d_out_b, "gate_ragged_plan: request with a null pointer");
        reqs.push_back(cbs::GateReq{q.d_a, q.d_b, q.d_out_a, q.d_out_b, static_cast<uint32_t>(items), q.count});
        items += q.count;
    }
    CBS_CHECK_ARG(items < (uint64_t(1) << 31), "gate_ragged_plan: more than 2^31 ciphertexts");
    ctx->plan_reqs = static_cast<uint32_t>(reqs.size());
    ctx->plan_items = static_cast<uint32_t>(items);
    ctx->plan_grid = (grid_ctas == 0 || grid_ctas > items) ? static_cast<uint32_t>(items) : grid_ctas;
    if (reqs.empty()) return CBS_OK;
    CBS_CUDA_TRY(ctx->d_plan.alloc(reqs.size()));
    CBS_CUDA_TRY(cudaMemcpy(ctx->d_plan.p, reqs.data(), reqs.size() * sizeof(cbs::GateReq), cudaMemcpyHostToDevice));
    CBS_CUDA_TRY(ctx->d_plan_ext.alloc(static_cast<size_t>(items) * (ctx->p.N + 1)));
    return CBS_OK;
}

cbs_status cbs_gate_ragged_autotune(cbs_gate_context* ctx, uint32_t* chosen_grid, double* ms_out) {
    CBS_CHECK_ARG(ctx, "gate_ragged_autotune: null context");
    if (ctx->plan_items == 0) {
        set_error("gate_ragged_autotune: no plan (call cbs_gate_ragged_plan first)");
        return CBS_ERR_NOT_READY;
    }
    int dev = 0, sms = 0;
    CBS_CUDA_TRY(cudaGetDevice(&dev));
    CBS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t items = ctx->plan_items, keep = ctx->plan_grid;
    const uint32_t su = static_cast<uint32_t>(sms);
    const uint32_t cands[] = {items, 2 * su, 4 * su, 8 * su};
    cudaStream_t s = nullptr;
    CBS_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    double best_ms = 1e300;
    uint32_t best = keep;
    cbs_status st = CBS_OK;
    for (uint32_t g : cands) {
        if (ce != cudaSuccess || st != CBS_OK) break;
        ctx->plan_grid = g > items ? items : g;
        if ((st = cbs_gate_ragged_launch(ctx, reinterpret_cast<cbs_stream_t>(s)))) break;  // warm-up
        ce = cudaEventRecord(e0, s);
        if (ce == cudaSuccess && (st = cbs_gate_ragged_launch(ctx, reinterpret_cast<cbs_stream_t>(s)))) break;
        if (ce == cudaSuccess) ce = cudaEventRecord(e1, s);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
        float ms = 0;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
        if (ce == cudaSuccess && ms < best_ms) {
            best_ms = ms;
            best = ctx->plan_grid;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    ctx->plan_grid = (st == CBS_OK && ce == cudaSuccess) ? best : keep;
    if (st != CBS_OK) return st;
    if (ce != cudaSuccess) {
        set_error(std::string("gate_ragged_autotune: ") + cudaGetErrorString(ce));
        return CBS_ERR_CUDA;
    }
    if (chosen_grid) *chosen_grid = best;
    if (ms_out) *ms_out = best_ms;
    return CBS_OK;
}

cbs_status cbs_gate_ragged_launch(cbs_gate_context* ctx, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "gate_ragged_launch: null context");
    if (ctx->plan_items == 0) return CBS_OK;
    const cbs_gate_params& p = ctx->p;
    cbs::GateArgs a{};
    if (cbs_status st = gate_fill_keys(ctx, a)) return st;
    a.gate = -1;
    a.n = p.n;
    a.levels = p.levels;
    a.bg_bits = p.bg_bits;
    a.ext = ctx->d_plan_ext.p;
    a.reqs = ctx->d_plan.p;
    a.num_reqs = ctx->plan_reqs;
    a.items = ctx->plan_items;
    a.levels_tv = 1;
    a.mu[0] = 1u << 29;
    CBS_CUDA_TRY(cbs::gate_blind_rotate(a, p.N, ctx->plan_grid, stream));
    const dim3 grid(ctx->plan_items, (p.n + 1 + 255) / 256);
    cbs::k_gate_keyswitch<<<grid, 256, (p.N + 1) * sizeof(uint32_t), stream>>>(
        static_cast<const uint32_t*>(a.ext), ctx->d_ksk.p, p.n, p.N, p.ks_base_bits, p.ks_levels, nullptr, nullptr,
        a.reqs, a.num_reqs);
    CBS_LAUNCH_CHECK();
    return CBS_OK;
}

}  // extern "C"
