// fft_ops.cuh -- element operations shared by the FP64 FFT kernels: reduction of an
// integer-valued double mod Q, balanced gadget digits by the offset trick, and the twist
// factors of the folded negacyclic transform.
#pragma once

#include "fft_core.cuh"
#include "fft_kernels.cuh"

namespace cbs {

// bit mask of the LWE coefficients in grouped key kk of a group of mb (the subset order of the
// grouped keys: mb = 2: {0} {1} {0,1}; mb = 3: {0} {1} {2} {0,1} {0,2} {1,2} {0,1,2}; mb = 4,
// the staged grouping: {0} {1} {2} {3} {0,1} {0,2} {1,2} {0,1,2})
__host__ __device__ constexpr uint32_t mb_key_mask(int mb, uint32_t kk) {
    if (mb == 2) return kk == 0 ? 1u : (kk == 1 ? 2u : 3u);
    if (mb == 4) return kk < 4 ? (1u << kk) : (kk == 4 ? 3u : (kk == 5 ? 5u : (kk == 6 ? 6u : 7u)));
    return kk < 3 ? (1u << kk) : (kk == 3 ? 3u : (kk == 4 ? 5u : (kk == 5 ? 6u : 7u)));
}

// grouped keys per group of mb coefficients: 2^mb - 1 subsets (mb = 2, 3); 8 for the staged mb = 4
__host__ __device__ constexpr uint32_t mb_group_keys(int mb) { return mb == 4 ? 8u : (1u << mb) - 1u; }

// LWE coefficients per step of a group (the staged mb = 4 runs steps of 3 and 1)
__host__ __device__ constexpr int mb_step_coefs(int mb) { return mb == 4 ? 3 : mb; }

// v mod Q, v the FP64 value of an integer-valued product (|v| < 2^90), computed in FP64:
// k = rint(v / Q), r = v - k*q_hi - k*q_lo with two fused multiply-adds.  The two roundings of
// r (|r| < 2Q < 2^55) add at most +-8 to the result, far below the FFT's own rounding error.
__device__ __forceinline__ uint64_t double_to_mod(double v, const FftKeyArgs& f, uint64_t Q) {
    const double k = rint(v * f.inv_q);
    double r = fma(-k, f.q_hi, v);
    r = fma(-k, f.q_lo, r);
    int64_t i = __double2ll_rn(r);
    if (i < 0) i += static_cast<int64_t>(Q);
    if (i < 0) i += static_cast<int64_t>(Q);
    if (i >= static_cast<int64_t>(Q)) i -= static_cast<int64_t>(Q);
    return static_cast<uint64_t>(i);
}

// v - rint(v / Q) Q as an int64, v the FP64 value of an integer-valued product (|v| < 2^90):
// within Q/2 + 2^37 of zero (the quotient's rounding can be off by one near a half-integer).
__device__ __forceinline__ int64_t centred_residue(double v, const FftKeyArgs& f) {
    const double k = rint(v * f.inv_q);
    double r = fma(-k, f.q_hi, v);
    r = fma(-k, f.q_lo, r);
    return __double2ll_rn(r);
}

// y + t brought back into the window [lo, lo + Q) = [lo, hi), for y in the window and |t| < Q/2
// + 2^37 (so one correction by +-Q suffices)
__device__ __forceinline__ int64_t offset_add(int64_t y, int64_t t, int64_t lo, int64_t hi, int64_t Q) {
    int64_t s = y + t;
    s = (s < lo) ? s + Q : s;
    return (s >= hi) ? s - Q : s;
}

// Balanced base-2^gbits digits of the prepared value v, all at once: adding
// O = sum_k 2^(gbits-1) 2^(gbits k) makes every digit field non-negative, so digit k is field
// k of v + O minus 2^(gbits-1).  This is the unique balanced representation of v modulo
// 2^(gbits digits) with digits in [-2^(gbits-1), 2^(gbits-1)), i.e. what peel_digit yields
// with the final carry dropped.
__device__ __forceinline__ int32_t balanced_digit(int64_t w, int gbits, uint32_t k) {
    const uint32_t field = static_cast<uint32_t>(static_cast<uint64_t>(w) >> (gbits * k)) & ((1u << gbits) - 1u);
    return static_cast<int32_t>(field) - (1 << (gbits - 1));
}

// gadget_prepare(x) + offset for x in [0, Q): centre, round away the ign low bits, add the
// digit offset.  The sum is non-negative because the offset times 2^ign is at least Q / 2.
__device__ __forceinline__ int64_t prepared_offset(uint64_t x, uint64_t Q, uint64_t qhalf, uint64_t round_c, int ign) {
    uint64_t t = x + round_c;
    if (x >= qhalf) t -= Q;
    return static_cast<int64_t>(t >> ign);
}

__device__ __forceinline__ uint32_t pack_digits(int32_t re, int32_t im) {
    return (static_cast<uint32_t>(re) & 0xffffu) | (static_cast<uint32_t>(im) << 16);
}

// zeta^e from the half table: register slot j of the first/last pass holds e = tid + j*M/8,
// so e < M/2 exactly for j < 4; above, zeta^e = i * conj(zeta^(M-e)) = swapped components.
template <int LOGM>
__device__ __forceinline__ double2 twist_at(const double2* tws, int j, uint32_t e) {
    if (j < 4) return tws[e];
    const double2 t = tws[(1u << LOGM) - e];
    return make_double2(t.y, t.x);
}

// zeta^m for zeta = exp(i pi / N), m in [0, 2N), from the half twist table (zeta^r for
// r <= N/4): m = q N/2 + r gives zeta^m = i^q zeta^r, and for r > N/4,
// zeta^r = i conj(zeta^(N/2 - r)) (the swapped components of entry N/2 - r).
template <int LOGN>
__device__ __forceinline__ double2 zeta_pow(const double2* tws, uint32_t m) {
    constexpr uint32_t N = 1u << LOGN;
    const uint32_t q = m >> (LOGN - 1), r = m & (N / 2 - 1);
    const bool up = r > N / 4;
    const double2 t = tws[up ? N / 2 - r : r];
    const double c = up ? t.y : t.x, s = up ? t.x : t.y;
    const double x = (q & 1) ? s : c, y = (q & 1) ? c : s;
    return make_double2((q == 1 || q == 2) ? -x : x, (q >= 2) ? -y : y);
}

// Register slot j of thread t in a forward transform's output (M = N/2 points, M/8 threads,
// slot s = 8t + j, bit-reversed order) holds the evaluation at psi_s = zeta^(4 rev(s) + 1).
// rev(s) = rev3(j) M/8 + rev(t) over log2(M/8) bits, so psi_s^a = zeta^(a e_t + a rev3(j) N/4)
// with e_t = 4 rev(t) + 1: mult_base() gives a e_t mod 2N once per step, slot_exp() the
// exponent of slot j.
template <int LOGN>
__device__ __forceinline__ uint32_t mult_base(uint32_t t, uint32_t a) {
    constexpr int TB = LOGN - 4;  // log2(M/8)
    const uint32_t rt = __brev(t) >> (32 - TB);
    return (a * (4 * rt + 1)) & ((2u << LOGN) - 1);
}
template <int LOGN>
__device__ __forceinline__ uint32_t slot_exp(uint32_t base, uint32_t a, int j) {
    const uint32_t r3 = ((j & 1) << 2) | (j & 2) | ((j >> 2) & 1);
    return (base + ((a * r3) & 7u) * ((1u << LOGN) / 4)) & ((2u << LOGN) - 1);
}

__device__ __forceinline__ int64_t prepared_offset(uint64_t x, const DigitPrep& g) {
    return prepared_offset(x, g.q, g.qhalf, g.round_c, g.ign);
}

// x in [0, Q) as the centred value, in FP64
__device__ __forceinline__ double centred_double(uint64_t x, uint64_t Q, uint64_t qhalf) {
    return static_cast<double>(x >= qhalf ? static_cast<int64_t>(x) - static_cast<int64_t>(Q)
                                          : static_cast<int64_t>(x));
}

// The biased digit fields (digit + 2^(gbits-1)) of one folded pair (a_e, a_(e+M)): packed in
// one 32-bit word for digits of up to 15 bits (re in the low half-word), two words for wider
// digits (the 2 x 18-bit gadget).
template <bool WIDE>
struct DigitPair {
    using T = uint32_t;
    __device__ static __forceinline__ T pack(uint32_t re, uint32_t im) { return re | (im << 16); }
    __device__ static __forceinline__ double2 unpack(T v, int32_t bias) {
        return make_double2(static_cast<double>(static_cast<int32_t>(v & 0xffffu) - bias),
                            static_cast<double>(static_cast<int32_t>(v >> 16) - bias));
    }
};
template <>
struct DigitPair<true> {
    using T = uint2;
    __device__ static __forceinline__ T pack(uint32_t re, uint32_t im) { return make_uint2(re, im); }
    __device__ static __forceinline__ double2 unpack(T v, int32_t bias) {
        return make_double2(static_cast<double>(static_cast<int32_t>(v.x) - bias),
                            static_cast<double>(static_cast<int32_t>(v.y) - bias));
    }
};

// gadget digits wider than the packed 16-bit fields take the two-word form
__host__ __device__ constexpr bool wide_digits(int gbits) { return gbits > 15; }

template <int LOGN>
struct BrFftCfg {
    static constexpr uint32_t T = (1u << LOGN) / 8;
    static constexpr int MIN_BLOCKS = LOGN <= 10 ? 4 : (LOGN == 11 ? 2 : 1);
};

}  // namespace cbs
