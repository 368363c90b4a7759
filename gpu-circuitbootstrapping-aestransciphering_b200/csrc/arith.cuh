// arith.cuh -- 64-bit modular arithmetic for sm_100a.
//
// Same arithmetic contract as the reference's include/uintmodmath.cuh and
// include/butterfly.cuh: values mod a single prime q < 2^62, Shoup products with a
// precomputed quotient w' = floor(w * 2^64 / q), lazy ranges [0, 2q) / [0, 4q)
// inside transforms, fully reduced [0, q) at every API boundary.
#pragma once

#include <cstdint>

namespace cbs {

__device__ __forceinline__ uint64_t csub(uint64_t x, uint64_t q) {
    const uint64_t t = x - q;
    return (static_cast<int64_t>(t) < 0) ? x : t;
}

__device__ __forceinline__ uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) { return csub(a + b, q); }

__device__ __forceinline__ uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) {
    const uint64_t t = a - b;
    return (a < b) ? t + q : t;
}

// x * w mod q in [0, 2q) for any x < 2^64 (Shoup, lazy)
__device__ __forceinline__ uint64_t mul_shoup_lazy(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
    const uint64_t hi = __umul64hi(x, ws);
    return x * w - hi * q;
}

__device__ __forceinline__ uint64_t mul_shoup(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
    return csub(mul_shoup_lazy(x, w, ws, q), q);
}

// 128-bit helpers
struct u128 {
    uint64_t lo, hi;
};

__device__ __forceinline__ u128 mul_wide(uint64_t a, uint64_t b) { return {a * b, __umul64hi(a, b)}; }

__device__ __forceinline__ void add_wide(u128& acc, u128 v) {
    asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;" : "+l"(acc.lo), "+l"(acc.hi) : "l"(v.lo), "l"(v.hi));
}

// Barrett reduction of a 128-bit value x < q * 2^64 with ratio = floor(2^128 / q) (two words),
// the constant Phantom stores in DModulus::const_ratio (src/host/modulus.h).
__device__ __forceinline__ uint64_t barrett_reduce_128(u128 x, uint64_t q, uint64_t r0, uint64_t r1) {
    // floor(x * ratio / 2^128), keeping the words that matter
    const uint64_t a_hi_r0_hi = __umul64hi(x.lo, r0);
    u128 t1 = mul_wide(x.lo, r1);
    u128 t2 = mul_wide(x.hi, r0);
    // middle word sum
    uint64_t mid = t1.lo, carry;
    asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, 0, 0;" : "+l"(mid), "=l"(carry) : "l"(a_hi_r0_hi));
    uint64_t mid2 = mid;
    uint64_t carry2;
    asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, 0, 0;" : "+l"(mid2), "=l"(carry2) : "l"(t2.lo));
    const uint64_t quot = x.hi * r1 + t1.hi + t2.hi + carry + carry2;
    const uint64_t r = x.lo - quot * q;
    return csub(r, q);
}

// Montgomery product x * k' * 2^-64 mod q in [0, 2q) for x < q, k' < q (k' = k * 2^64 mod q
// gives x * k): keys stored in Montgomery form need no Shoup companion, so a MAC reads one
// word per key coefficient.  qneg_inv = -q^-1 mod 2^64.
__device__ __forceinline__ uint64_t mont_mul_lazy(uint64_t x, uint64_t kp, uint64_t q, uint64_t qneg_inv) {
    const uint64_t lo = x * kp;
    const uint64_t hi = __umul64hi(x, kp);
    const uint64_t m = lo * qneg_inv;
    return hi + __umul64hi(m, q) + (lo != 0 ? 1ull : 0ull);
}

// s mod q for any s < 2^64 using the Shoup quotient of 1 (one_s = floor(2^64 / q))
__device__ __forceinline__ uint64_t reduce64(uint64_t s, uint64_t q, uint64_t one_s) {
    const uint64_t hi = __umul64hi(s, one_s);
    return csub(csub(s - hi * q, q), q);
}

// Montgomery-free exact product a * b mod q with a 128-bit intermediate (setup paths only).
__device__ __forceinline__ uint64_t mul_mod_barrett(uint64_t a, uint64_t b, uint64_t q, uint64_t r0, uint64_t r1) {
    return barrett_reduce_128(mul_wide(a, b), q, r0, r1);
}

// Signed gadget decomposition, the contract of bitwise/src/cirbts/kernel.cu:37-68
// (device_SignedDigitDecompose2): drop ign = logQ - digits*gbits low bits with a
// balanced rounding, then balanced base-2^gbits digits (least significant first);
// a final carry is discarded.  Digits are returned as signed integers.
struct Gadget {
    int gbits;
    int ign;
    uint64_t q;
};

__host__ __device__ inline Gadget make_gadget(uint64_t q, uint32_t base, uint32_t digits) {
    Gadget g;
    int gb = 0;
    while ((1u << gb) < base) ++gb;
    int logq = 0;
    while (logq < 64 && (q >> logq) != 0) ++logq;
    int ign = logq - static_cast<int>(digits) * gb;
    g.gbits = gb;
    g.ign = ign < 0 ? 0 : ign;
    g.q = q;
    return g;
}

// returns the centered value after dropping the ignored bits; digits are then peeled
// with peel_digit()
__device__ __forceinline__ int64_t gadget_prepare(uint64_t x, const Gadget& g) {
    const uint64_t qhalf = g.q >> 1;
    int64_t d = (x < qhalf) ? static_cast<int64_t>(x) : static_cast<int64_t>(x) - static_cast<int64_t>(g.q);
    if (g.ign != 0) {
        const int s = 64 - g.ign;
        const int64_t r = static_cast<int64_t>(static_cast<uint64_t>(d) << s) >> s;
        d = (d - r) >> g.ign;
    }
    return d;
}

__device__ __forceinline__ int32_t peel_digit(int64_t& d, int gbits) {
    const int s = 64 - gbits;
    const int64_t r = static_cast<int64_t>(static_cast<uint64_t>(d) << s) >> s;
    d = (d - r) >> gbits;
    return static_cast<int32_t>(r);
}

__device__ __forceinline__ uint64_t signed_to_mod(int64_t v, uint64_t q) {
    return v < 0 ? static_cast<uint64_t>(v + static_cast<int64_t>(q)) : static_cast<uint64_t>(v);
}

}  // namespace cbs
