// fp64_mod.cuh -- exact modular arithmetic on the FP64 pipe for primes below 2^50.
//
// The 64-bit Shoup / Barrett products of arith.cuh are emulated with 32-bit integer multiplies
// and bound the integer pipe while the FP64 pipe idles.  For q < 2^50 every residue, lazy value
// and constant is an integer below 2^53, held exactly in a double, and the modular product is
// computed exactly in doubles:
//   h = fl(v w), l = fma(v, w, -h)          (error-free product, Ogita-Rump-Oishi TwoProduct:
//                                            v w = h + l exactly)
//   k = rint(h * fl(1/q))                   (quotient estimate: |v w / q - k| <= 1/2 + 3 |v| 2^-53)
//   r = fma(-k, q, h) + l                    (= v w - k q exactly)
// fma(-k, q, h) is exact because its true value h - k q = r - l is an integer below 2^53 in
// magnitude; r is congruent to v w and |r| <= q (1/2 + 3 |v| 2^-53), i.e. below 0.875 q for
// |v| < 2^50 and below 2q for |v| < 2^52.  This is the floating-point quotient estimate of
// Shoup's MulMod (NTL) carried out entirely in doubles.
#pragma once

#include <cstdint>

namespace cbs {

struct DMod {
    double q, qinv;
};

__device__ __forceinline__ DMod dmod_of(uint64_t q) { return {static_cast<double>(q), 1.0 / static_cast<double>(q)}; }

// v w mod q, signed (see above), exact for |v| < 2^52 and 0 <= w < q < 2^50
__device__ __forceinline__ double dmulmod(double v, double w, const DMod& m) {
    const double h = __dmul_rn(v, w);
    const double l = __fma_rn(v, w, -h);
    const double k = rint(__dmul_rn(h, m.qinv));
    return __dadd_rn(__fma_rn(-k, m.q, h), l);
}

// x mod q in [-q/2 - 1, q/2 + 1] for |x| < 2^53
__device__ __forceinline__ double dreduce(double x, const DMod& m) {
    return __fma_rn(-rint(__dmul_rn(x, m.qinv)), m.q, x);
}

// the residue in [0, q) of an integer |x| < 2^53
__device__ __forceinline__ uint64_t dto_residue(double x, const DMod& m) {
    double r = dreduce(x, m);
    if (r < 0.0) r = __dadd_rn(r, m.q);
    return __double2ull_rn(r);
}

}  // namespace cbs
