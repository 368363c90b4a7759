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
__device__ __forceinline__ double2 mul_i(double2 v) { return make_double2(-v.y, v.x); }
__device__ __forceinline__ double2 mul_negi(double2 v) { return make_double2(v.y, -v.x); }

// the same operations in FP32 (the split-FP32 external product of the 32-bit torus)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csubd(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
    acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
}
__device__ __forceinline__ float2 mul_i(float2 v) { return make_float2(-v.y, v.x); }
__device__ __forceinline__ float2 mul_negi(float2 v) { return make_float2(v.y, -v.x); }

// Shared-memory swizzles of the transform buffers.  16-byte elements: e ^ ((e >> 3) & 7)
// makes every pass free of bank conflicts for M = 512 and 1024; 8-byte elements need the
// four-bit form e ^ ((e >> 3) & 15) (both permute the low four bits only, so they stay
// inside [0, M) and inside every aligned block of 16).
__device__ __forceinline__ uint32_t cswz(uint32_t e) { return e ^ ((e >> 3) & 7u); }
template <class C>
__device__ __forceinline__ uint32_t cswz_of(uint32_t e) {
    if constexpr (sizeof(C) == 8) return e ^ ((e >> 3) & 15u);
    else return cswz(e);
}

// DIF butterfly: (u, v) -> (u + v, (u - v) * w)
template <class C>
__device__ __forceinline__ void dif_bf(C& u, C& v, C w) {
    const C s = cadd(u, v);
    v = cmul(csubd(u, v), w);
    u = s;
}
// DIT butterfly (inverse of the above up to a factor 2): (p, s) -> (p + s*conj(w), p - s*conj(w))
template <class C>
__device__ __forceinline__ void dit_bf(C& p, C& s, C w) {
    const C t = cmulc(s, w);
    s = csubd(p, t);
    p = cadd(p, t);
}

// Twiddle tables of one transform length, kept in shared memory by the kernels:
//   [0, M/2)            tw[e] = exp(2*pi*i*e/M), read directly by the first pass (its index
//                       runs over consecutive e);
//   pass_off(p), p >= 1 the twiddles of pass p laid out [k][j0] (k = the butterfly's place in
//                       the pass, j0 = the thread's group), so the lanes of a warp read
//                       consecutive entries;
//   twist_off()         exp(i*pi*e/N) for e <= M/2 (e > M/2 uses zeta^(M-e) = i conj(zeta^e),
//                       i.e. the swapped components of entry M - e).
template <int LOGM>
struct FftTab {
    static constexpr uint32_t M = 1u << LOGM;
    using Pl = NttPlan<LOGM>;
    static constexpr uint32_t pass_m(int p) { return 1u << (3 * p); }
    static constexpr int pass_r(int p) { return p < Pl::P - 1 ? 3 : Pl::tail_r; }
    static constexpr uint32_t pass_size(int p) {
        return pass_r(p) == 3 ? 7 * (M / (8 * pass_m(p)))
                              : (pass_r(p) == 2 ? 3 * (M / (4 * pass_m(p))) : M / (2 * pass_m(p)));
    }
    static constexpr uint32_t pass_off(int p) {
        uint32_t o = M / 2;
        for (int k = 1; k < p; ++k) o += pass_size(k);
        return o;
    }
    static constexpr uint32_t twist_off() { return pass_off(Pl::P); }
    static constexpr uint32_t size() { return twist_off() + M / 2 + 1; }
};

// DIF pass over R stages starting at DFT half-size h = M / (2m).  COMPACT: tb is the pass's
// [k][j0] table; otherwise tb is tw, indexed directly.  Twiddles known to be 1 or i are
// applied without multiplications.
template <int LOGM, int R, bool COMPACT, class C>
__device__ __forceinline__ void dif_pass(C (&x)[8], uint32_t m, uint32_t tid, const C* tb) {
    constexpr uint32_t M = 1u << LOGM;
    const uint32_t h = M / (2 * m);
    if (R == 3) {
        const uint32_t q = h / 4, j0 = tid % q;
        if (COMPACT && q == 1) {  // h = 4: stage 1 twiddles 1, w8, i, w8^3; stage 2 1, i; stage 3 1
            {
                const C t = csubd(x[0], x[4]);
                x[0] = cadd(x[0], x[4]);
                x[4] = t;
            }
            dif_bf(x[1], x[5], tb[1]);
            {
                const C t = mul_i(csubd(x[2], x[6]));
                x[2] = cadd(x[2], x[6]);
                x[6] = t;
            }
            dif_bf(x[3], x[7], tb[3]);
            // stage 2: twiddle 1 on the slot pairs (0,2), (4,6) and i on (1,3), (5,7)
#pragma unroll
            for (int g = 0; g < 8; g += 4) {
                C t = csubd(x[g], x[g + 2]);
                x[g] = cadd(x[g], x[g + 2]);
                x[g + 2] = t;
                t = mul_i(csubd(x[g + 1], x[g + 3]));
                x[g + 1] = cadd(x[g + 1], x[g + 3]);
                x[g + 3] = t;
            }
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const C t = csubd(x[r], x[r + 1]);
                x[r] = cadd(x[r], x[r + 1]);
                x[r + 1] = t;
            }
            return;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) dif_bf(x[r], x[r + 4], COMPACT ? tb[r * q + j0] : tb[(j0 + r * q) * m]);
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const C w = COMPACT ? tb[4 * q + r * q + j0] : tb[(j0 + r * q) * 2 * m];
            dif_bf(x[r], x[r + 2], w);
            dif_bf(x[r + 4], x[r + 6], w);
        }
        if (COMPACT && q == 2) {  // h = 8: the last stage's twiddle is i^j0
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const C t = csubd(x[r], x[r + 1]);
                x[r] = cadd(x[r], x[r + 1]);
                x[r + 1] = j0 ? mul_i(t) : t;
            }
        } else {
            const C w = COMPACT ? tb[6 * q + j0] : tb[j0 * 4 * m];
#pragma unroll
            for (int r = 0; r < 8; r += 2) dif_bf(x[r], x[r + 1], w);
        }
    } else if (R == 2) {
        const uint32_t q = h / 2;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const uint32_t j0 = (2 * tid + hh) % q;
            C* v = x + 4 * hh;
            if (COMPACT && q == 1) {  // twiddles 1, i, 1
                C t = csubd(v[0], v[2]);
                v[0] = cadd(v[0], v[2]);
                v[2] = t;
                t = mul_i(csubd(v[1], v[3]));
                v[1] = cadd(v[1], v[3]);
                v[3] = t;
                t = csubd(v[0], v[1]);
                v[0] = cadd(v[0], v[1]);
                v[1] = t;
                t = csubd(v[2], v[3]);
                v[2] = cadd(v[2], v[3]);
                v[3] = t;
            } else {
                dif_bf(v[0], v[2], COMPACT ? tb[j0] : tb[j0 * m]);
                dif_bf(v[1], v[3], COMPACT ? tb[q + j0] : tb[(j0 + q) * m]);
                const C w = COMPACT ? tb[2 * q + j0] : tb[j0 * 2 * m];
                dif_bf(v[0], v[1], w);
                dif_bf(v[2], v[3], w);
            }
        }
    } else {
#pragma unroll
        for (int hh = 0; hh < 4; ++hh) {
            if (COMPACT && h == 1) {  // twiddle 1
                const C t = csubd(x[2 * hh], x[2 * hh + 1]);
                x[2 * hh] = cadd(x[2 * hh], x[2 * hh + 1]);
                x[2 * hh + 1] = t;
            } else {
                const uint32_t j0 = (4 * tid + hh) % h;
                dif_bf(x[2 * hh], x[2 * hh + 1], COMPACT ? tb[j0] : tb[j0 * m]);
            }
        }
    }
}

template <int LOGM, int R, bool COMPACT, class C>
__device__ __forceinline__ void dit_pass(C (&x)[8], uint32_t m, uint32_t tid, const C* tb) {
    constexpr uint32_t M = 1u << LOGM;
    const uint32_t h = M / (2 * m);
    if (R == 3) {
        const uint32_t q = h / 4, j0 = tid % q;
        if (COMPACT && q == 1) {
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const C t = x[r + 1];
                x[r + 1] = csubd(x[r], t);
                x[r] = cadd(x[r], t);
            }
#pragma unroll
            for (int g = 0; g < 8; g += 4) {  // twiddle 1 on (0,2), (4,6); i (conjugated) on (1,3), (5,7)
                C t = x[g + 2];
                x[g + 2] = csubd(x[g], t);
                x[g] = cadd(x[g], t);
                t = mul_negi(x[g + 3]);
                x[g + 3] = csubd(x[g + 1], t);
                x[g + 1] = cadd(x[g + 1], t);
            }
            {
                const C t = x[4];
                x[4] = csubd(x[0], t);
                x[0] = cadd(x[0], t);
            }
            dit_bf(x[1], x[5], tb[1]);
            {
                const C t = mul_negi(x[6]);
                x[6] = csubd(x[2], t);
                x[2] = cadd(x[2], t);
            }
            dit_bf(x[3], x[7], tb[3]);
            return;
        }
        if (COMPACT && q == 2) {
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const C t = j0 ? mul_negi(x[r + 1]) : x[r + 1];
                x[r + 1] = csubd(x[r], t);
                x[r] = cadd(x[r], t);
            }
        } else {
            const C w = COMPACT ? tb[6 * q + j0] : tb[j0 * 4 * m];
#pragma unroll
            for (int r = 0; r < 8; r += 2) dit_bf(x[r], x[r + 1], w);
        }
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const C w = COMPACT ? tb[4 * q + r * q + j0] : tb[(j0 + r * q) * 2 * m];
            dit_bf(x[r], x[r + 2], w);
            dit_bf(x[r + 4], x[r + 6], w);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) dit_bf(x[r], x[r + 4], COMPACT ? tb[r * q + j0] : tb[(j0 + r * q) * m]);
    } else if (R == 2) {
        const uint32_t q = h / 2;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const uint32_t j0 = (2 * tid + hh) % q;
            C* v = x + 4 * hh;
            if (COMPACT && q == 1) {
                C t = v[1];
                v[1] = csubd(v[0], t);
                v[0] = cadd(v[0], t);
                t = v[3];
                v[3] = csubd(v[2], t);
                v[2] = cadd(v[2], t);
                t = v[2];
                v[2] = csubd(v[0], t);
                v[0] = cadd(v[0], t);
                t = mul_negi(v[3]);
                v[3] = csubd(v[1], t);
                v[1] = cadd(v[1], t);
            } else {
                const C w = COMPACT ? tb[2 * q + j0] : tb[j0 * 2 * m];
                dit_bf(v[0], v[1], w);
                dit_bf(v[2], v[3], w);
                dit_bf(v[0], v[2], COMPACT ? tb[j0] : tb[j0 * m]);
                dit_bf(v[1], v[3], COMPACT ? tb[q + j0] : tb[(j0 + q) * m]);
            }
        }
    } else {
#pragma unroll
        for (int hh = 0; hh < 4; ++hh) {
            if (COMPACT && h == 1) {
                const C t = x[2 * hh + 1];
                x[2 * hh + 1] = csubd(x[2 * hh], t);
                x[2 * hh] = cadd(x[2 * hh], t);
            } else {
                const uint32_t j0 = (4 * tid + hh) % h;
                dit_bf(x[2 * hh], x[2 * hh + 1], COMPACT ? tb[j0] : tb[j0 * m]);
            }
        }
    }
}

// Shared-memory exchanges: the elements a thread reads before pass p (forward) lie in one
// block of the previous pass, written by the (M >> 3(p-1)) / 8 threads of that block; when
// that group fits in a warp (aligned, consecutive threads) the exchange needs only
// __syncwarp().  Before inverse pass p the writers are the (M >> 3p) / 8 threads of the
// reader's own pass-p block.  Other exchanges call the caller's barrier over the M/8
// threads of this transform.  Every pass writes exactly the set it read, and the sets of a
// pass partition [0, M), so no write needs a barrier before it.
template <int LOGM>
constexpr bool fwd_exchange_in_warp(int p) {
    return ((1u << LOGM) >> (3 * (p - 1))) / 8 <= 32;
}
template <int LOGM>
constexpr bool inv_exchange_in_warp(int p) {
    return ((1u << LOGM) >> (3 * p)) / 8 <= 32;
}

// Forward FFT of one folded, twisted polynomial by M/8 threads.  tab: the FftTab layout (in
// shared memory); load(j, e) returns z_e for register slot j (e < M); on return x[j] holds
// spectrum slot 8*tid + j.  sm: M elements of shared memory, which the caller must not let
// other threads of the group still be reading when this is entered; bar() synchronises the
// M/8 threads of the transform.
template <int LOGM, class Load, class Bar, class C>
__device__ __forceinline__ void fft_forward_to_regs(C* sm, uint32_t tid, const C* tab, Load load, C (&x)[8], Bar bar) {
    using Pl = NttPlan<LOGM>;
    using Tb = FftTab<LOGM>;
    static_assert(Pl::P >= 2, "fft needs M >= 64");
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = load(j, pass_index<LOGM, 3>(1u, tid, j));
    dif_pass<LOGM, 3, false>(x, 1u, tid, tab);
#pragma unroll
    for (int p = 1; p < Pl::P; ++p) {
#pragma unroll
        for (int j = 0; j < 8; ++j) sm[cswz_of<C>(pass_index<LOGM, 3>(1u << (3 * (p - 1)), tid, j))] = x[j];
        if (fwd_exchange_in_warp<LOGM>(p)) __syncwarp();
        else bar();
        const uint32_t m = 1u << (3 * p);
        if (p < Pl::P - 1) {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = sm[cswz_of<C>(pass_index<LOGM, 3>(m, tid, j))];
            dif_pass<LOGM, 3, true>(x, m, tid, tab + Tb::pass_off(p));
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = sm[cswz_of<C>(pass_index<LOGM, Pl::tail_r>(m, tid, j))];
            dif_pass<LOGM, Pl::tail_r, true>(x, m, tid, tab + Tb::pass_off(p));
        }
    }
}

// Two independent forward FFTs in lockstep (the same M/8 threads, separate exchange buffers
// sm0 / sm1): each pass's butterflies of both transforms interleave, which doubles the
// independent FP64 work between exchanges, and the two transforms share every barrier.
template <int LOGM, class Load0, class Load1, class Bar, class C>
__device__ __forceinline__ void fft_forward2_to_regs(C* sm0, C* sm1, uint32_t tid, const C* tab, Load0 load0,
                                                     Load1 load1, C (&x0)[8], C (&x1)[8], Bar bar) {
    using Pl = NttPlan<LOGM>;
    using Tb = FftTab<LOGM>;
    static_assert(Pl::P >= 2, "fft needs M >= 64");
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t e = pass_index<LOGM, 3>(1u, tid, j);
        x0[j] = load0(j, e);
        x1[j] = load1(j, e);
    }
    dif_pass<LOGM, 3, false>(x0, 1u, tid, tab);
    dif_pass<LOGM, 3, false>(x1, 1u, tid, tab);
#pragma unroll
    for (int p = 1; p < Pl::P; ++p) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t e = cswz_of<C>(pass_index<LOGM, 3>(1u << (3 * (p - 1)), tid, j));
            sm0[e] = x0[j];
            sm1[e] = x1[j];
        }
        if (fwd_exchange_in_warp<LOGM>(p)) __syncwarp();
        else bar();
        const uint32_t m = 1u << (3 * p);
        if (p < Pl::P - 1) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t e = cswz_of<C>(pass_index<LOGM, 3>(m, tid, j));
                x0[j] = sm0[e];
                x1[j] = sm1[e];
            }
            dif_pass<LOGM, 3, true>(x0, m, tid, tab + Tb::pass_off(p));
            dif_pass<LOGM, 3, true>(x1, m, tid, tab + Tb::pass_off(p));
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t e = cswz_of<C>(pass_index<LOGM, Pl::tail_r>(m, tid, j));
                x0[j] = sm0[e];
                x1[j] = sm1[e];
            }
            dif_pass<LOGM, Pl::tail_r, true>(x0, m, tid, tab + Tb::pass_off(p));
            dif_pass<LOGM, Pl::tail_r, true>(x1, m, tid, tab + Tb::pass_off(p));
        }
    }
}

// Inverse FFT (without the 1/M factor) from the thread's spectrum slots 8*tid + j in x;
// store(j, e, v) receives element e < M in natural order (register slot j, a compile-time
// constant after unrolling, so callers can keep per-slot results in registers).  Same
// shared-memory contract and barrier as the forward transform; on return other threads of
// the group may still be reading sm.
template <int LOGM, class Store, class Bar, class C>
__device__ __forceinline__ void fft_inverse_from_regs(C* sm, uint32_t tid, const C* tab, C (&x)[8], Store store,
                                                      Bar bar) {
    using Pl = NttPlan<LOGM>;
    using Tb = FftTab<LOGM>;
    constexpr uint32_t mt = 1u << (3 * (Pl::P - 1));
    dit_pass<LOGM, Pl::tail_r, true>(x, mt, tid, tab + Tb::pass_off(Pl::P - 1));
#pragma unroll
    for (int j = 0; j < 8; ++j) sm[cswz_of<C>(pass_index<LOGM, Pl::tail_r>(mt, tid, j))] = x[j];
    if (inv_exchange_in_warp<LOGM>(Pl::P - 2)) __syncwarp();
    else bar();
#pragma unroll
    for (int p = Pl::P - 2; p >= 0; --p) {
        const uint32_t m = 1u << (3 * p);
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = sm[cswz_of<C>(pass_index<LOGM, 3>(m, tid, j))];
        if (p == 0) dit_pass<LOGM, 3, false>(x, m, tid, tab);
        else dit_pass<LOGM, 3, true>(x, m, tid, tab + Tb::pass_off(p));
        if (p > 0) {
            // each pass reads and writes its own per-thread set and the sets partition [0, M), so
            // the write needs no barrier; the read of pass p - 1 does
#pragma unroll
            for (int j = 0; j < 8; ++j) sm[cswz_of<C>(pass_index<LOGM, 3>(m, tid, j))] = x[j];
            if (inv_exchange_in_warp<LOGM>(p - 1)) __syncwarp();
            else bar();
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) store(j, pass_index<LOGM, 3>(1u, tid, j), x[j]);
}

}  // namespace cbs
