// cbs_kernels.cuh -- launch interfaces of the fused circuit-bootstrapping, CMux and
// extraction kernels (implemented in cbs_kernels.cu, lut_kernels.cu, extract_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "arith.cuh"

namespace cbs {

struct RingTables {
    const uint64_t* rp;
    const uint64_t* rps;
    const uint64_t* irp;
    const uint64_t* irps;
    uint64_t q;
    uint64_t n_inv, n_inv_s;
    uint64_t ratio0, ratio1;  // floor(2^128 / q)
    uint64_t qneg_inv;        // -q^-1 mod 2^64 (Montgomery)
    uint64_t one_s;           // floor(2^64 / q)
};

struct BlindRotateArgs {
    RingTables t;
    const uint64_t* a;       // [batch][a_stride] LWE masks mod q_lwe
    const uint64_t* b;       // [batch]
    uint32_t a_stride;
    uint32_t n;              // LWE dimension (blind-rotation steps)
    uint64_t q_lwe;
    uint32_t bitwidth;       // special mod-switch granularity log2
    const uint64_t* tv;      // [N] test vector, coefficient domain
    const uint64_t* bsk;     // [n][2*digits][2][N] NTT domain, Montgomery form
    Gadget g;                // blind-rotation gadget
    uint32_t digits;
    uint32_t num_lut;
    const uint64_t* gadd;    // [num_lut] (gpow[j] >> 1) * N^-1 mod Q
    uint64_t* mv_out;        // [batch][num_lut][2][N] NTT domain (MV RLWEs after finalize)
    uint32_t schedule;       // FFT grouped form: CBS_BR_SCHEDULE_* (0 = the tuned / default choice)
};

struct TraceArgs {
    RingTables t;
    const uint64_t* mv;      // [count][2][N] NTT domain
    uint64_t* rgsw;          // [count][2][2][N] NTT domain
    const uint32_t* maps;    // [rounds][N] NTT-domain automorphism permutations
    uint32_t rounds;
    const uint64_t* ht_key;  // [rounds][digits_ht][2][N] NTT domain, Montgomery form
    const uint64_t* ss_key;  // [digits_ss][2][N] NTT domain, Montgomery form
    Gadget g_ht, g_ss;
    uint32_t digits_ht, digits_ss;
};

struct CmuxLevelArgs {
    RingTables t;
    const uint64_t* in;           // level input: [sets][in_count][2][N]
    uint64_t in_lut_stride;       // words between input sets
    const uint32_t* lut_sel;      // input set of each LUT (level 0: table id); null = the LUT index
    uint64_t* out;                // [luts][in_count/2][2][N]
    uint32_t in_count;
    const uint64_t* rgsw_all;     // CBS output [bits][digits][2][2][N]
    uint64_t rgsw_stride;         // words per bit
    const uint32_t* ctrl_bits;    // [luts][8] bit index of the control for each level
    uint32_t level;
    Gadget g;
    uint32_t digits;
};

// bitwise/src/cirbts/kernel.cu:7316-7326 device_SpecialMS_IndexPos (same FP64 expression
// and rounding): round v * 2N / (q * 2^bw) to an integer, times 2^bw, mod 2N
__device__ __forceinline__ uint32_t special_ms_f(uint64_t v, uint32_t two_n, uint64_t q, uint32_t bitwidth) {
    const uint64_t shift = (bitwidth < 63u) ? (1ull << bitwidth) : 0ull;
    if (shift == 0ull || two_n == 0u || q == 0) return 0u;
    const double scale = static_cast<double>(two_n) / (static_cast<double>(q) * static_cast<double>(shift));
    const double x = static_cast<double>(v) * scale;
    const uint64_t r = __double2ull_rd(x + 0.5);
    return static_cast<uint32_t>((r * shift) & (static_cast<uint64_t>(two_n) - 1ull));
}

// coefficient i of X^{-e} p (e in [0, 2N))
template <uint32_t N>
__device__ __forceinline__ uint64_t rot_neg(const uint64_t* p, uint32_t e, uint32_t i, uint64_t q) {
    const uint32_t s = (i + e) & (2 * N - 1);
    const uint64_t v = (s < N) ? p[s] : p[s - N];
    return (s < N) ? v : (v ? q - v : 0);
}

cudaError_t launch_blind_rotate(const BlindRotateArgs& a, uint32_t N, uint32_t batch, cudaStream_t s);
cudaError_t launch_trace_schemeswitch(const TraceArgs& a, uint32_t N, uint32_t count, cudaStream_t s);
cudaError_t launch_cmux_level(const CmuxLevelArgs& a, uint32_t N, uint32_t luts, cudaStream_t s);

}  // namespace cbs
