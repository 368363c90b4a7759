// ntt_core.cuh -- register-blocked negacyclic NTT for one polynomial per CTA on sm_100a.
//
// Transform contract (identical outputs to the reference's src/ntt/ntt_1d.cu):
//   forward: Cooley-Tukey stages m = 1, 2, ..., N/2; group k of stage m uses the twiddle
//            tw[m + k] from Phantom's bit-reversed power table (src/host/ntt.cu:11-56);
//            output in bit-reversed evaluation order, fully reduced to [0, q).
//   inverse: Gentleman-Sande stages m = N/2 ... 1 with itw[m + k]; the n^-1 factor is
//            applied on the last stage (x by n_inv, y through itw[1] which has n^-1
//            folded in), output fully reduced.
// Design: N/8 threads per polynomial, 8 coefficients per thread in registers, three
// stages per shared-memory round trip (radix-8 passes, a radix-4/2 tail), XOR-swizzled
// shared memory (i ^ ((i >> 3) & 15)) so every pass is free of bank conflicts, lazy
// Harvey butterflies with Shoup twiddles.  One __syncthreads per pass boundary: each pass
// reads and writes the same per-thread index set, and the sets partition [0, N).
#pragma once

#include "arith.cuh"

namespace cbs {

__device__ __forceinline__ uint32_t swz(uint32_t i) { return i ^ ((i >> 3) & 15u); }

// forward (CT) butterfly, inputs < 4q, outputs < 4q
__device__ __forceinline__ void ct_bf(uint64_t& x, uint64_t& y, uint64_t w, uint64_t ws, uint64_t q2, uint64_t q) {
    const uint64_t t = mul_shoup_lazy(y, w, ws, q);  // [0, 2q)
    x = csub(x, q2);                                 // [0, 2q)
    y = x + q2 - t;
    x = x + t;
}

// inverse (GS) butterfly, inputs < 2q, outputs < 2q
__device__ __forceinline__ void gs_bf(uint64_t& x, uint64_t& y, uint64_t w, uint64_t ws, uint64_t q2, uint64_t q) {
    const uint64_t t = x + q2 - y;
    x = csub(x + y, q2);
    y = mul_shoup_lazy(t, w, ws, q);
}

template <int LOGN>
struct NttPlan {
    static constexpr int N = 1 << LOGN;
    static constexpr int T = N / 8;               // threads per polynomial
    static constexpr int P = (LOGN + 2) / 3;      // passes
    static constexpr int tail_r = LOGN - 3 * (P - 1);
    static constexpr int radix(int p) { return p < P - 1 ? 3 : tail_r; }
};

// Index of register slot j of thread tid in the pass that starts (forward) or ends
// (inverse) at stage m and covers R stages.
template <int LOGN, int R>
__device__ __forceinline__ uint32_t pass_index(uint32_t m, uint32_t tid, int j) {
    constexpr uint32_t N = 1u << LOGN;
    const uint32_t blk = N / m;  // elements per group block
    if (R == 3) {
        const uint32_t q4 = N / (8 * m);
        const uint32_t k = tid / q4, b = tid % q4;
        return k * blk + b + j * q4;
    } else if (R == 2) {
        const uint32_t half = N / (4 * m);
        const uint32_t s = 2 * tid + (j >> 2);
        const uint32_t k = s / half, b = s % half;
        return k * blk + b + (j & 3) * half;
    } else {
        const uint32_t t = N / (2 * m);
        const uint32_t s = 4 * tid + (j >> 1);
        const uint32_t k = s / t, b = s % t;
        return k * blk + b + (j & 1) * t;
    }
}

template <int LOGN, int R>
__device__ __forceinline__ uint32_t pass_group(uint32_t m, uint32_t tid, int set) {
    constexpr uint32_t N = 1u << LOGN;
    if (R == 3) return tid / (N / (8 * m));
    if (R == 2) return (2 * tid + set) / (N / (4 * m));
    return (4 * tid + set) / (N / (2 * m));
}

template <int LOGN, int R>
__device__ __forceinline__ void fwd_pass(uint64_t (&x)[8], uint32_t m, uint32_t tid, const uint64_t* __restrict__ tw,
                                         const uint64_t* __restrict__ tws, uint64_t q) {
    const uint64_t q2 = q << 1;
    if (R == 3) {
        const uint32_t k = pass_group<LOGN, 3>(m, tid, 0);
        const uint32_t i1 = m + k;
        {
            const uint64_t w = __ldg(tw + i1), ws = __ldg(tws + i1);
#pragma unroll
            for (int j = 0; j < 4; ++j) ct_bf(x[j], x[j + 4], w, ws, q2, q);
        }
        {
            const uint64_t w0 = __ldg(tw + 2 * i1), w0s = __ldg(tws + 2 * i1);
            const uint64_t w1 = __ldg(tw + 2 * i1 + 1), w1s = __ldg(tws + 2 * i1 + 1);
            ct_bf(x[0], x[2], w0, w0s, q2, q);
            ct_bf(x[1], x[3], w0, w0s, q2, q);
            ct_bf(x[4], x[6], w1, w1s, q2, q);
            ct_bf(x[5], x[7], w1, w1s, q2, q);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t ti = 4 * i1 + j;
            ct_bf(x[2 * j], x[2 * j + 1], __ldg(tw + ti), __ldg(tws + ti), q2, q);
        }
    } else if (R == 2) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t k = pass_group<LOGN, 2>(m, tid, h);
            const uint32_t i1 = m + k;
            const uint64_t w = __ldg(tw + i1), ws = __ldg(tws + i1);
            uint64_t* v = x + 4 * h;
            ct_bf(v[0], v[2], w, ws, q2, q);
            ct_bf(v[1], v[3], w, ws, q2, q);
            ct_bf(v[0], v[1], __ldg(tw + 2 * i1), __ldg(tws + 2 * i1), q2, q);
            ct_bf(v[2], v[3], __ldg(tw + 2 * i1 + 1), __ldg(tws + 2 * i1 + 1), q2, q);
        }
    } else {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const uint32_t k = pass_group<LOGN, 1>(m, tid, h);
            const uint32_t i1 = m + k;
            ct_bf(x[2 * h], x[2 * h + 1], __ldg(tw + i1), __ldg(tws + i1), q2, q);
        }
    }
}

template <int LOGN, int R>
__device__ __forceinline__ void inv_pass(uint64_t (&x)[8], uint32_t m, uint32_t tid, const uint64_t* __restrict__ tw,
                                         const uint64_t* __restrict__ tws, uint64_t q) {
    const uint64_t q2 = q << 1;
    if (R == 3) {
        const uint32_t k = pass_group<LOGN, 3>(m, tid, 0);
        const uint32_t i1 = m + k;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t ti = 4 * i1 + j;
            gs_bf(x[2 * j], x[2 * j + 1], __ldg(tw + ti), __ldg(tws + ti), q2, q);
        }
        {
            const uint64_t w0 = __ldg(tw + 2 * i1), w0s = __ldg(tws + 2 * i1);
            const uint64_t w1 = __ldg(tw + 2 * i1 + 1), w1s = __ldg(tws + 2 * i1 + 1);
            gs_bf(x[0], x[2], w0, w0s, q2, q);
            gs_bf(x[1], x[3], w0, w0s, q2, q);
            gs_bf(x[4], x[6], w1, w1s, q2, q);
            gs_bf(x[5], x[7], w1, w1s, q2, q);
        }
        {
            const uint64_t w = __ldg(tw + i1), ws = __ldg(tws + i1);
#pragma unroll
            for (int j = 0; j < 4; ++j) gs_bf(x[j], x[j + 4], w, ws, q2, q);
        }
    } else if (R == 2) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t k = pass_group<LOGN, 2>(m, tid, h);
            const uint32_t i1 = m + k;
            uint64_t* v = x + 4 * h;
            gs_bf(v[0], v[1], __ldg(tw + 2 * i1), __ldg(tws + 2 * i1), q2, q);
            gs_bf(v[2], v[3], __ldg(tw + 2 * i1 + 1), __ldg(tws + 2 * i1 + 1), q2, q);
            const uint64_t w = __ldg(tw + i1), ws = __ldg(tws + i1);
            gs_bf(v[0], v[2], w, ws, q2, q);
            gs_bf(v[1], v[3], w, ws, q2, q);
        }
    } else {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const uint32_t k = pass_group<LOGN, 1>(m, tid, h);
            const uint32_t i1 = m + k;
            gs_bf(x[2 * h], x[2 * h + 1], __ldg(tw + i1), __ldg(tws + i1), q2, q);
        }
    }
}

// Forward NTT of one polynomial held by the CTA's first NttPlan::T threads.
// load(i) supplies input coefficient i (< 4q); store(j, i, v) receives the fully reduced
// output at bit-reversed slot i (register slot j of this thread).  sm: N words of shared memory.  The caller must
// __syncthreads() before reusing sm.
template <int LOGN, class Load, class Store>
__device__ __forceinline__ void ntt_forward_cta(uint64_t* sm, uint32_t tid, const uint64_t* __restrict__ tw,
                                                const uint64_t* __restrict__ tws, uint64_t q, Load load, Store store) {
    using Pl = NttPlan<LOGN>;
    static_assert(Pl::P >= 2, "ntt_forward_cta needs N >= 64");
    uint64_t x[8];
    // first radix-8 pass straight from the loader
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = load(pass_index<LOGN, 3>(1u, tid, j));
    fwd_pass<LOGN, 3>(x, 1u, tid, tw, tws, q);
#pragma unroll
    for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGN, 3>(1u, tid, j))] = x[j];
    __syncthreads();
    // middle radix-8 passes (kept rolled: lower register pressure inside fused kernels)
#pragma unroll 1
    for (int p = 1; p < Pl::P - 1; ++p) {
        const uint32_t m = 1u << (3 * p);
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGN, 3>(m, tid, j))];
        fwd_pass<LOGN, 3>(x, m, tid, tw, tws, q);
#pragma unroll
        for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGN, 3>(m, tid, j))] = x[j];
        __syncthreads();
    }
    // tail pass to the store
    {
        constexpr uint32_t m = 1u << (3 * (Pl::P - 1));
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGN, Pl::tail_r>(m, tid, j))];
        fwd_pass<LOGN, Pl::tail_r>(x, m, tid, tw, tws, q);
        const uint64_t q2 = q << 1;
#pragma unroll
        for (int j = 0; j < 8; ++j) store(j, pass_index<LOGN, Pl::tail_r>(m, tid, j), csub(csub(x[j], q2), q));
    }
}

// Inverse NTT (n^-1 included) of one polynomial; load(j, i) supplies bit-reversed slot i
// (< 2q) for register slot j; store(i, v) receives coefficient i fully reduced.
template <int LOGN, class Load, class Store>
__device__ __forceinline__ void ntt_inverse_cta(uint64_t* sm, uint32_t tid, const uint64_t* __restrict__ itw,
                                                const uint64_t* __restrict__ itws, uint64_t n_inv, uint64_t n_inv_s,
                                                uint64_t q, Load load, Store store) {
    using Pl = NttPlan<LOGN>;
    static_assert(Pl::P >= 2, "ntt_inverse_cta needs N >= 64");
    uint64_t x[8];
    {
        constexpr uint32_t m = 1u << (3 * (Pl::P - 1));
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = load(j, pass_index<LOGN, Pl::tail_r>(m, tid, j));
        inv_pass<LOGN, Pl::tail_r>(x, m, tid, itw, itws, q);
#pragma unroll
        for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGN, Pl::tail_r>(m, tid, j))] = x[j];
        __syncthreads();
    }
#pragma unroll 1
    for (int p = Pl::P - 2; p >= 1; --p) {
        const uint32_t m = 1u << (3 * p);
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGN, 3>(m, tid, j))];
        inv_pass<LOGN, 3>(x, m, tid, itw, itws, q);
#pragma unroll
        for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGN, 3>(m, tid, j))] = x[j];
        __syncthreads();
    }
    // last pass (stages 4, 2, 1): x-halves (index < N/2) take n^-1 here, y-halves have it
    // folded into itw[1]
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGN, 3>(1u, tid, j))];
    inv_pass<LOGN, 3>(x, 1u, tid, itw, itws, q);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t idx = pass_index<LOGN, 3>(1u, tid, j);
        uint64_t v = csub(x[j], q);
        if (j < 4) v = mul_shoup(v, n_inv, n_inv_s, q);
        store(idx, v);
    }
}

}  // namespace cbs

namespace cbs {

// Register-resident forms used by the fused kernels.  For N = 1024, 2048, 4096 the last
// forward pass (and the first inverse pass) gives thread tid the eight consecutive
// bit-reversed slots 8*tid + j, j = 0..7; these helpers expose them in x[j].
template <int LOGN>
__device__ __forceinline__ uint32_t owned_slot(uint32_t tid, int j) {
    return 8u * tid + static_cast<uint32_t>(j);
}

template <int LOGN, class Load>
__device__ __forceinline__ void ntt_forward_to_regs(uint64_t* sm, uint32_t tid, const uint64_t* __restrict__ tw,
                                                    const uint64_t* __restrict__ tws, uint64_t q, Load load,
                                                    uint64_t (&out)[8]) {
    ntt_forward_cta<LOGN>(sm, tid, tw, tws, q, load, [&](int j, uint32_t, uint64_t v) { out[j] = v; });
}

// Inverse NTT starting from the thread's owned slots in x (values < 2q).
template <int LOGN, class Store>
__device__ __forceinline__ void ntt_inverse_from_regs(uint64_t* sm, uint32_t tid, const uint64_t* __restrict__ itw,
                                                      const uint64_t* __restrict__ itws, uint64_t n_inv,
                                                      uint64_t n_inv_s, uint64_t q, const uint64_t (&x)[8],
                                                      Store store) {
    ntt_inverse_cta<LOGN>(sm, tid, itw, itws, n_inv, n_inv_s, q, [&](int j, uint32_t) { return x[j]; }, store);
}

}  // namespace cbs
