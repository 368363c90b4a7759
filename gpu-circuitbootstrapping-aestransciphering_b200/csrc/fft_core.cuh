// fft_core.cuh -- register-blocked FP64 complex FFT of length M = N/2 for negacyclic
// products over Z[X]/(X^N + 1) on sm_100a.
//
// Folding (the scheme of bitwise/src/fft.cu:3614-3755, written from the mathematics): a
// real length-N polynomial a is evaluated at the odd powers zeta^(4k+1), zeta = e^(i*pi/N),
// as a cyclic length-M DFT of z_j = (a_j + i*a_(j+M)) * zeta^j; products of evaluations are
// evaluations of the negacyclic product, and the inverse DFT, the untwist by zeta^-j and the
// unfold (real part -> c_j, imaginary part -> c_(j+M)) recover it.
// Forward: decimation in frequency, natural order in, bit-reversed spectrum out; inverse:
// decimation in time, bit-reversed in, natural out (no bit-reversal pass either way, the
// spectra of keys are stored in the same bit-reversed order).  M/8 threads, eight complex
// values per thread, three stages per shared-memory round trip; the 16-byte elements are
// swizzled e ^ ((e >> 3) & 7), which makes every pass free of bank conflicts for M = 1024.
// The thread/index structure is the one of the integer NTT (ntt_core.cuh): the pass that
// starts at DFT half-size h uses the sets of the NTT pass at stage m = M / (2h).
#pragma once

#include "ntt_core.cuh"

namespace cbs {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csubd(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
// acc += a * b
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}

__device__ __forceinline__ uint32_t cswz(uint32_t e) { return e ^ ((e >> 3) & 7u); }

// DIF butterfly: (u, v) -> (u + v, (u - v) * w)
__device__ __forceinline__ void dif_bf(double2& u, double2& v, double2 w) {
    const double2 s = cadd(u, v);
    v = cmul(csubd(u, v), w);
    u = s;
}
// DIT butterfly (inverse of the above up to a factor 2): (p, s) -> (p + s*conj(w), p - s*conj(w))
__device__ __forceinline__ void dit_bf(double2& p, double2& s, double2 w) {
    const double2 t = cmulc(s, w);
    s = csubd(p, t);
    p = cadd(p, t);
}

// tw[e] = exp(2*pi*i*e / M), e < M/2
template <int LOGM, int R>
__device__ __forceinline__ void dif_pass(double2 (&x)[8], uint32_t m, uint32_t tid, const double2* __restrict__ tw) {
    constexpr uint32_t M = 1u << LOGM;
    const uint32_t h = M / (2 * m);
    if (R == 3) {
        const uint32_t q = h / 4, j0 = tid % q;
#pragma unroll
        for (int r = 0; r < 4; ++r) dif_bf(x[r], x[r + 4], __ldg(tw + (j0 + r * q) * m));
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const double2 w = __ldg(tw + (j0 + r * q) * 2 * m);
            dif_bf(x[r], x[r + 2], w);
            dif_bf(x[r + 4], x[r + 6], w);
        }
        const double2 w = __ldg(tw + j0 * 4 * m);
#pragma unroll
        for (int r = 0; r < 8; r += 2) dif_bf(x[r], x[r + 1], w);
    } else if (R == 2) {
        const uint32_t q = h / 2;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const uint32_t j0 = (2 * tid + hh) % q;
            double2* v = x + 4 * hh;
            dif_bf(v[0], v[2], __ldg(tw + j0 * m));
            dif_bf(v[1], v[3], __ldg(tw + (j0 + q) * m));
            const double2 w = __ldg(tw + j0 * 2 * m);
            dif_bf(v[0], v[1], w);
            dif_bf(v[2], v[3], w);
        }
    } else {
#pragma unroll
        for (int hh = 0; hh < 4; ++hh) {
            const uint32_t j0 = (4 * tid + hh) % h;
            dif_bf(x[2 * hh], x[2 * hh + 1], __ldg(tw + j0 * m));
        }
    }
}

template <int LOGM, int R>
__device__ __forceinline__ void dit_pass(double2 (&x)[8], uint32_t m, uint32_t tid, const double2* __restrict__ tw) {
    constexpr uint32_t M = 1u << LOGM;
    const uint32_t h = M / (2 * m);
    if (R == 3) {
        const uint32_t q = h / 4, j0 = tid % q;
        {
            const double2 w = __ldg(tw + j0 * 4 * m);
#pragma unroll
            for (int r = 0; r < 8; r += 2) dit_bf(x[r], x[r + 1], w);
        }
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const double2 w = __ldg(tw + (j0 + r * q) * 2 * m);
            dit_bf(x[r], x[r + 2], w);
            dit_bf(x[r + 4], x[r + 6], w);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) dit_bf(x[r], x[r + 4], __ldg(tw + (j0 + r * q) * m));
    } else if (R == 2) {
        const uint32_t q = h / 2;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const uint32_t j0 = (2 * tid + hh) % q;
            double2* v = x + 4 * hh;
            const double2 w = __ldg(tw + j0 * 2 * m);
            dit_bf(v[0], v[1], w);
            dit_bf(v[2], v[3], w);
            dit_bf(v[0], v[2], __ldg(tw + j0 * m));
            dit_bf(v[1], v[3], __ldg(tw + (j0 + q) * m));
        }
    } else {
#pragma unroll
        for (int hh = 0; hh < 4; ++hh) {
            const uint32_t j0 = (4 * tid + hh) % h;
            dit_bf(x[2 * hh], x[2 * hh + 1], __ldg(tw + j0 * m));
        }
    }
}

// Forward FFT of one folded, twisted polynomial by the first M/8 threads of the CTA.
// load(e) returns z_e (e < M); on return x[j] holds spectrum slot 8*tid + j.
// sm: M double2 of shared memory; the caller __syncthreads() before reusing it.
template <int LOGM, class Load>
__device__ __forceinline__ void fft_forward_to_regs(double2* sm, uint32_t tid, const double2* __restrict__ tw,
                                                    Load load, double2 (&x)[8]) {
    using Pl = NttPlan<LOGM>;
    static_assert(Pl::P >= 2, "fft needs M >= 64");
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = load(pass_index<LOGM, 3>(1u, tid, j));
    dif_pass<LOGM, 3>(x, 1u, tid, tw);
#pragma unroll
    for (int p = 1; p < Pl::P; ++p) {
#pragma unroll
        for (int j = 0; j < 8; ++j) sm[cswz(pass_index<LOGM, 3>(1u << (3 * (p - 1)), tid, j))] = x[j];
        __syncthreads();
        const uint32_t m = 1u << (3 * p);
        if (p < Pl::P - 1) {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = sm[cswz(pass_index<LOGM, 3>(m, tid, j))];
            dif_pass<LOGM, 3>(x, m, tid, tw);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = sm[cswz(pass_index<LOGM, Pl::tail_r>(m, tid, j))];
            dif_pass<LOGM, Pl::tail_r>(x, m, tid, tw);
        }
    }
}

// Inverse FFT (without the 1/M factor) from the thread's spectrum slots 8*tid + j in x;
// store(j, e, v) receives element e < M in natural order (register slot j, a compile-time
// constant after unrolling, so callers can keep per-slot results in registers).
template <int LOGM, class Store>
__device__ __forceinline__ void fft_inverse_from_regs(double2* sm, uint32_t tid, const double2* __restrict__ tw,
                                                      double2 (&x)[8], Store store) {
    using Pl = NttPlan<LOGM>;
    constexpr uint32_t mt = 1u << (3 * (Pl::P - 1));
    dit_pass<LOGM, Pl::tail_r>(x, mt, tid, tw);
#pragma unroll
    for (int j = 0; j < 8; ++j) sm[cswz(pass_index<LOGM, Pl::tail_r>(mt, tid, j))] = x[j];
    __syncthreads();
#pragma unroll
    for (int p = Pl::P - 2; p >= 0; --p) {
        const uint32_t m = 1u << (3 * p);
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = sm[cswz(pass_index<LOGM, 3>(m, tid, j))];
        dit_pass<LOGM, 3>(x, m, tid, tw);
        if (p > 0) {
            // each pass reads and writes its own per-thread set, and the sets partition [0, M)
#pragma unroll
            for (int j = 0; j < 8; ++j) sm[cswz(pass_index<LOGM, 3>(m, tid, j))] = x[j];
            __syncthreads();
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) store(j, pass_index<LOGM, 3>(1u, tid, j), x[j]);
}

}  // namespace cbs
