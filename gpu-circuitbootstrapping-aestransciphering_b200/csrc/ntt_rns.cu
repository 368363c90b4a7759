// ntt_rns.cu -- multi-prime negacyclic NTT for N = 2^10 .. 2^17 (Phantom's RNS NTT).
//
// Same transform as src/ntt/fntt_2d.cu / intt_2d.cu (nwt_2d_radix8_forward_inplace and
// nwt_2d_radix8_backward_inplace): per limb a Cooley-Tukey negacyclic NTT with Phantom's
// bit-reversed twiddle table of that limb's prime, bit-reversed output, n^-1 folded into the
// last inverse stage; outputs fully reduced, bit-identical.
//
// Structure: N = 2^L1 * 2^L2 with L2 = 8.  The first L1 forward stages only mix elements
// congruent mod 2^L2 ("columns"): stage m, group k of the full transform is stage m, group k
// of a 2^L1-point transform of column c, twiddle index m + k.  The last L2 stages stay inside
// rows of 2^L2 consecutive elements: for row R, local stage m and group k use twiddle index
// m*(2^L1 + R) + k of the full table.  Each phase is one kernel of register-blocked
// sub-transforms (8 coefficients per thread, radix-8 passes through swizzled shared memory),
// so a limb crosses HBM twice per transform.  Columns: a CTA takes 16 adjacent columns and
// its threads interleave columns so every global access is a 128-byte run; rows: 16 rows of
// 256 contiguous words per CTA.  Intermediate values stay lazy (< 4q forward, < 2q
// inverse); the second kernel reduces fully.  When every prime of the chain is below 2^50
// the same kernels run on the FP64 pipe (exact products in doubles, see below).
#include <atomic>

#include "async_copy.cuh"
#include "common.cuh"
#include "fp64_mod.cuh"
#include "ntt_core.cuh"
#include "ntt_rns.cuh"

namespace cbs {

// forward pass with an explicit twiddle base: i1 = base + k
template <int LOGS, int R>
__device__ __forceinline__ void fwd_pass_b(uint64_t (&x)[8], uint32_t m, uint32_t base, uint32_t tid,
                                           const uint64_t* __restrict__ tw, const uint64_t* __restrict__ tws,
                                           uint64_t q) {
    const uint64_t q2 = q << 1;
    if (R == 3) {
        const uint32_t i1 = base + pass_group<LOGS, 3>(m, tid, 0);
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
            const uint32_t i1 = base + pass_group<LOGS, 2>(m, tid, h);
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
            const uint32_t i1 = base + pass_group<LOGS, 1>(m, tid, h);
            ct_bf(x[2 * h], x[2 * h + 1], __ldg(tw + i1), __ldg(tws + i1), q2, q);
        }
    }
}

template <int LOGS, int R>
__device__ __forceinline__ void inv_pass_b(uint64_t (&x)[8], uint32_t m, uint32_t base, uint32_t tid,
                                           const uint64_t* __restrict__ tw, const uint64_t* __restrict__ tws,
                                           uint64_t q) {
    const uint64_t q2 = q << 1;
    if (R == 3) {
        const uint32_t i1 = base + pass_group<LOGS, 3>(m, tid, 0);
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
            const uint32_t i1 = base + pass_group<LOGS, 2>(m, tid, h);
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
            const uint32_t i1 = base + pass_group<LOGS, 1>(m, tid, h);
            gs_bf(x[2 * h], x[2 * h + 1], __ldg(tw + i1), __ldg(tws + i1), q2, q);
        }
    }
}

// 2^LOGS-point forward sub-transform of one group; twb(m) gives the twiddle base of local
// stage m; load(e), store(e, v) address the group's elements (lazy values)
template <int LOGS, class TwB, class Load, class Store>
__device__ __forceinline__ void sub_fwd(uint64_t* sm, uint32_t gt, const uint64_t* __restrict__ tw,
                                        const uint64_t* __restrict__ tws, uint64_t q, TwB twb, Load load,
                                        Store store) {
    using Pl = NttPlan<LOGS>;
    uint64_t x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = load(pass_index<LOGS, 3>(1u, gt, j));
    fwd_pass_b<LOGS, 3>(x, 1u, twb(1u), gt, tw, tws, q);
#pragma unroll
    for (int p = 1; p < Pl::P; ++p) {
#pragma unroll
        for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGS, 3>(1u << (3 * (p - 1)), gt, j))] = x[j];
        __syncthreads();
        const uint32_t m = 1u << (3 * p);
        if (p < Pl::P - 1) {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGS, 3>(m, gt, j))];
            fwd_pass_b<LOGS, 3>(x, m, twb(m), gt, tw, tws, q);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGS, Pl::tail_r>(m, gt, j))];
            fwd_pass_b<LOGS, Pl::tail_r>(x, m, twb(m), gt, tw, tws, q);
        }
    }
    constexpr uint32_t mt = 1u << (3 * (Pl::P - 1));
#pragma unroll
    for (int j = 0; j < 8; ++j) store(pass_index<LOGS, Pl::tail_r>(mt, gt, j), x[j]);
}

template <int LOGS, class TwB, class Load, class Store>
__device__ __forceinline__ void sub_inv(uint64_t* sm, uint32_t gt, const uint64_t* __restrict__ tw,
                                        const uint64_t* __restrict__ tws, uint64_t q, TwB twb, Load load,
                                        Store store) {
    using Pl = NttPlan<LOGS>;
    constexpr uint32_t mt = 1u << (3 * (Pl::P - 1));
    uint64_t x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = load(pass_index<LOGS, Pl::tail_r>(mt, gt, j));
    inv_pass_b<LOGS, Pl::tail_r>(x, mt, twb(mt), gt, tw, tws, q);
#pragma unroll
    for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGS, Pl::tail_r>(mt, gt, j))] = x[j];
    __syncthreads();
#pragma unroll
    for (int p = Pl::P - 2; p >= 0; --p) {
        const uint32_t m = 1u << (3 * p);
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGS, 3>(m, gt, j))];
        inv_pass_b<LOGS, 3>(x, m, twb(m), gt, tw, tws, q);
        if (p > 0) {
#pragma unroll
            for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGS, 3>(m, gt, j))] = x[j];
            __syncthreads();
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) store(pass_index<LOGS, 3>(1u, gt, j), x[j], j);
}


// ---------------------------------------------------------------------------------------------
// FP64-pipe form (primes below 2^50): the exact modular products of fp64_mod.cuh.  Values are
// signed and lazy: each radix-8 pass first reduces its 8 inputs to |x| <= q/2 + 1, after which
// three forward stages grow them to at most 2q + 4 and three inverse stages to at most
// 4q + 8, far inside the exact range.  The twiddles are the same tables converted to doubles;
// results are the integer path's residues, bit for bit.
__device__ __forceinline__ void ct_bf_d(double& x, double& y, double w, const DMod& m) {
    const double t = dmulmod(y, w, m);
    y = __dsub_rn(x, t);
    x = __dadd_rn(x, t);
}

__device__ __forceinline__ void gs_bf_d(double& x, double& y, double w, const DMod& m) {
    const double t = __dsub_rn(x, y);
    x = __dadd_rn(x, y);
    y = dmulmod(t, w, m);
}

// the passes of fwd_pass_b / inv_pass_b with double values and twiddles; inputs reduced first
template <int LOGS, int R>
__device__ __forceinline__ void fwd_pass_d(double (&x)[8], uint32_t m, uint32_t base, uint32_t tid,
                                           const double* __restrict__ tw, const DMod& md) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = dreduce(x[j], md);
    if (R == 3) {
        const uint32_t i1 = base + pass_group<LOGS, 3>(m, tid, 0);
        {
            const double w = __ldg(tw + i1);
#pragma unroll
            for (int j = 0; j < 4; ++j) ct_bf_d(x[j], x[j + 4], w, md);
        }
        {
            const double w0 = __ldg(tw + 2 * i1), w1 = __ldg(tw + 2 * i1 + 1);
            ct_bf_d(x[0], x[2], w0, md);
            ct_bf_d(x[1], x[3], w0, md);
            ct_bf_d(x[4], x[6], w1, md);
            ct_bf_d(x[5], x[7], w1, md);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) ct_bf_d(x[2 * j], x[2 * j + 1], __ldg(tw + 4 * i1 + j), md);
    } else if (R == 2) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t i1 = base + pass_group<LOGS, 2>(m, tid, h);
            const double w = __ldg(tw + i1);
            double* v = x + 4 * h;
            ct_bf_d(v[0], v[2], w, md);
            ct_bf_d(v[1], v[3], w, md);
            ct_bf_d(v[0], v[1], __ldg(tw + 2 * i1), md);
            ct_bf_d(v[2], v[3], __ldg(tw + 2 * i1 + 1), md);
        }
    } else {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const uint32_t i1 = base + pass_group<LOGS, 1>(m, tid, h);
            ct_bf_d(x[2 * h], x[2 * h + 1], __ldg(tw + i1), md);
        }
    }
}

template <int LOGS, int R>
__device__ __forceinline__ void inv_pass_d(double (&x)[8], uint32_t m, uint32_t base, uint32_t tid,
                                           const double* __restrict__ tw, const DMod& md) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = dreduce(x[j], md);
    if (R == 3) {
        const uint32_t i1 = base + pass_group<LOGS, 3>(m, tid, 0);
#pragma unroll
        for (int j = 0; j < 4; ++j) gs_bf_d(x[2 * j], x[2 * j + 1], __ldg(tw + 4 * i1 + j), md);
        {
            const double w0 = __ldg(tw + 2 * i1), w1 = __ldg(tw + 2 * i1 + 1);
            gs_bf_d(x[0], x[2], w0, md);
            gs_bf_d(x[1], x[3], w0, md);
            gs_bf_d(x[4], x[6], w1, md);
            gs_bf_d(x[5], x[7], w1, md);
        }
        {
            const double w = __ldg(tw + i1);
#pragma unroll
            for (int j = 0; j < 4; ++j) gs_bf_d(x[j], x[j + 4], w, md);
        }
    } else if (R == 2) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint32_t i1 = base + pass_group<LOGS, 2>(m, tid, h);
            double* v = x + 4 * h;
            gs_bf_d(v[0], v[1], __ldg(tw + 2 * i1), md);
            gs_bf_d(v[2], v[3], __ldg(tw + 2 * i1 + 1), md);
            const double w = __ldg(tw + i1);
            gs_bf_d(v[0], v[2], w, md);
            gs_bf_d(v[1], v[3], w, md);
        }
    } else {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const uint32_t i1 = base + pass_group<LOGS, 1>(m, tid, h);
            gs_bf_d(x[2 * h], x[2 * h + 1], __ldg(tw + i1), md);
        }
    }
}

// sub_fwd_d with two hooks: after_loads() runs after the first CTA barrier (every initial load
// of every thread has completed), before_store() just before the outputs are stored
template <int LOGS, class TwB, class Load, class Store, class AfterLoads, class BeforeStore>
__device__ __forceinline__ void sub_fwd_d_hooked(double* sm, uint32_t gt, const double* __restrict__ tw,
                                                 const DMod& md, TwB twb, Load load, Store store,
                                                 AfterLoads after_loads, BeforeStore before_store) {
    using Pl = NttPlan<LOGS>;
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = load(pass_index<LOGS, 3>(1u, gt, j));
    fwd_pass_d<LOGS, 3>(x, 1u, twb(1u), gt, tw, md);
#pragma unroll
    for (int p = 1; p < Pl::P; ++p) {
#pragma unroll
        for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGS, 3>(1u << (3 * (p - 1)), gt, j))] = x[j];
        __syncthreads();
        if (p == 1) after_loads();
        const uint32_t m = 1u << (3 * p);
        if (p < Pl::P - 1) {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGS, 3>(m, gt, j))];
            fwd_pass_d<LOGS, 3>(x, m, twb(m), gt, tw, md);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGS, Pl::tail_r>(m, gt, j))];
            fwd_pass_d<LOGS, Pl::tail_r>(x, m, twb(m), gt, tw, md);
        }
    }
    constexpr uint32_t mt = 1u << (3 * (Pl::P - 1));
    before_store();
#pragma unroll
    for (int j = 0; j < 8; ++j) store(pass_index<LOGS, Pl::tail_r>(mt, gt, j), x[j]);
}

template <int LOGS, class TwB, class Load, class Store>
__device__ __forceinline__ void sub_fwd_d(double* sm, uint32_t gt, const double* __restrict__ tw, const DMod& md,
                                          TwB twb, Load load, Store store) {
    sub_fwd_d_hooked<LOGS>(sm, gt, tw, md, twb, load, store, []() {}, []() {});
}

template <int LOGS, class TwB, class Load, class Store>
__device__ __forceinline__ void sub_inv_d(double* sm, uint32_t gt, const double* __restrict__ tw, const DMod& md,
                                          TwB twb, Load load, Store store) {
    using Pl = NttPlan<LOGS>;
    constexpr uint32_t mt = 1u << (3 * (Pl::P - 1));
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = load(pass_index<LOGS, Pl::tail_r>(mt, gt, j));
    inv_pass_d<LOGS, Pl::tail_r>(x, mt, twb(mt), gt, tw, md);
#pragma unroll
    for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGS, Pl::tail_r>(mt, gt, j))] = x[j];
    __syncthreads();
#pragma unroll
    for (int p = Pl::P - 2; p >= 0; --p) {
        const uint32_t m = 1u << (3 * p);
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = sm[swz(pass_index<LOGS, 3>(m, gt, j))];
        inv_pass_d<LOGS, 3>(x, m, twb(m), gt, tw, md);
        if (p > 0) {
#pragma unroll
            for (int j = 0; j < 8; ++j) sm[swz(pass_index<LOGS, 3>(m, gt, j))] = x[j];
            __syncthreads();
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) store(pass_index<LOGS, 3>(1u, gt, j), x[j], j);
}

constexpr int kL2 = 8;            // row stages (rows of 256 words)
constexpr uint32_t kGroups = 16;  // sub-transforms per CTA

// column groups are padded by one word so the 16 interleaved columns of a warp hit 16
// different banks
template <int L1>
constexpr uint32_t col_stride() {
    return (1u << L1) + 1;
}

__device__ __forceinline__ uint64_t* limb_ptr(uint64_t* data, const RnsNttArgs& a, uint32_t limb_flat,
                                              uint32_t log_n) {
    const uint32_t poly = limb_flat / a.limbs, limb = limb_flat % a.limbs;
    const uint32_t slot = a.limb_slot ? a.limb_slot[limb] : limb;
    return data + static_cast<size_t>(poly) * a.poly_stride + (static_cast<size_t>(slot) << log_n);
}

// source of the first phase: in (out-of-place) or data
__device__ __forceinline__ const uint64_t* src_ptr(uint64_t* data, const RnsNttArgs& a, uint32_t limb_flat,
                                                   uint32_t log_n) {
    if (!a.in) return limb_ptr(data, a, limb_flat, log_n);
    const uint32_t poly = limb_flat / a.limbs, limb = limb_flat % a.limbs;
    const uint32_t slot = a.limb_slot ? a.limb_slot[limb] : limb;
    return a.in + static_cast<size_t>(poly) * a.in_poly_stride + (static_cast<size_t>(slot) << log_n);
}

// forward phase 1: columns (2^L1 points each, stride 2^L2), lazy output (FP: signed lazy
// doubles written in place, read back by the row phase)
template <int L1, bool FP>
__global__ void __launch_bounds__(kGroups * (1 << L1) / 8) k_rns_fwd_cols(uint64_t* __restrict__ data,
                                                                         const RnsNttArgs a) {
    constexpr uint32_t ROW = 1u << kL2;
    extern __shared__ uint64_t sm[];
    const uint32_t tid = threadIdx.x;
    const uint32_t g = tid % kGroups, gt = tid / kGroups;  // lanes interleave columns
    const uint32_t colblk = blockIdx.x % (ROW / kGroups);
    const uint32_t limb_flat = blockIdx.x / (ROW / kGroups);  // poly * limbs + limb
    const uint32_t prime = a.limb_prime[limb_flat % a.limbs];
    const size_t N = size_t(1) << (L1 + kL2);
    const uint64_t* tw = a.tw + prime * N;
    const uint64_t* tws = a.tws + prime * N;
    const uint64_t q = a.q[prime];
    uint64_t* poly = limb_ptr(data, a, limb_flat, L1 + kL2) + colblk * kGroups + g;
    const uint64_t* src = src_ptr(data, a, limb_flat, L1 + kL2) + colblk * kGroups + g;
    if constexpr (FP) {
        double* dpoly = reinterpret_cast<double*>(poly);
        sub_fwd_d<L1>(
            reinterpret_cast<double*>(sm) + g * col_stride<L1>(), gt, a.twd + prime * N, dmod_of(q),
            [](uint32_t m) { return m; }, [&](uint32_t e) { return __ull2double_rn(src[e * ROW]); },
            [&](uint32_t e, double v) { dpoly[e * ROW] = v; });
    } else {
        sub_fwd<L1>(
            sm + g * col_stride<L1>(), gt, tw, tws, q, [](uint32_t m) { return m; },
            [&](uint32_t e) { return src[e * ROW]; }, [&](uint32_t e, uint64_t v) { poly[e * ROW] = v; });
    }
}

// forward phase 2: rows (256 contiguous words), full reduction, optional moddown epilogue
template <int L1, int EPI, bool FP>
__global__ void __launch_bounds__(kGroups * 32) k_rns_fwd_rows(uint64_t* __restrict__ data, const RnsNttArgs a) {
    constexpr uint32_t ROW = 1u << kL2, ROWS = 1u << L1;
    extern __shared__ uint64_t sm[];
    const uint32_t tid = threadIdx.x;
    const uint32_t g = tid / 32, gt = tid % 32;
    const uint32_t rowblk = blockIdx.x % (ROWS / kGroups);
    const uint32_t limb_flat = blockIdx.x / (ROWS / kGroups);
    const uint32_t prime = a.limb_prime[limb_flat % a.limbs];
    const size_t N = size_t(1) << (L1 + kL2);
    const uint64_t* tw = a.tw + prime * N;
    const uint64_t* tws = a.tws + prime * N;
    const uint64_t q = a.q[prime], q2 = q << 1;
    const uint32_t R = rowblk * kGroups + g;
    uint64_t* row = limb_ptr(data, a, limb_flat, L1 + kL2) + static_cast<size_t>(R) * ROW;
    if constexpr (FP) {
        const DMod md = dmod_of(q);
        const double* drow = reinterpret_cast<const double*>(row);
        double* dsm = reinterpret_cast<double*>(sm) + g * ROW;
        const double* twd = a.twd + prime * N;
        if (EPI == 0) {
            sub_fwd_d<kL2>(
                dsm, gt, twd, md, [&](uint32_t m) { return m * (ROWS + R); }, [&](uint32_t e) { return drow[e]; },
                [&](uint32_t e, double v) { row[e] = dto_residue(v, md); });
        } else {
            const uint32_t poly = limb_flat / a.limbs, limb = limb_flat % a.limbs;
            const size_t off = (static_cast<size_t>(limb) << (L1 + kL2)) + static_cast<size_t>(R) * ROW;
            const uint64_t* cx = a.epi_cx + poly * a.epi_cx_stride + off;
            uint64_t* dst = a.epi_dst + poly * a.epi_dst_stride + off;
            const uint64_t f = a.epi_f[limb], fs = a.epi_fs[limb];
            sub_fwd_d<kL2>(
                dsm, gt, twd, md, [&](uint32_t m) { return m * (ROWS + R); }, [&](uint32_t e) { return drow[e]; },
                [&](uint32_t e, double dv) {
                    const uint64_t v = dto_residue(dv, md);
                    uint64_t r = mul_shoup(sub_mod(cx[e], v, q), f, fs, q);
                    if (EPI == 2) r = add_mod(dst[e], r, q);
                    dst[e] = r;
                });
        }
        return;
    }
    if (EPI == 0) {
        sub_fwd<kL2>(
            sm + g * ROW, gt, tw, tws, q, [&](uint32_t m) { return m * (ROWS + R); },
            [&](uint32_t e) { return row[e]; }, [&](uint32_t e, uint64_t v) { row[e] = csub(csub(v, q2), q); });
    } else {
        const uint32_t poly = limb_flat / a.limbs, limb = limb_flat % a.limbs;
        const size_t off = (static_cast<size_t>(limb) << (L1 + kL2)) + static_cast<size_t>(R) * ROW;
        const uint64_t* cx = a.epi_cx + poly * a.epi_cx_stride + off;
        uint64_t* dst = a.epi_dst + poly * a.epi_dst_stride + off;
        const uint64_t f = a.epi_f[limb], fs = a.epi_fs[limb];
        sub_fwd<kL2>(
            sm + g * ROW, gt, tw, tws, q, [&](uint32_t m) { return m * (ROWS + R); },
            [&](uint32_t e) { return row[e]; },
            [&](uint32_t e, uint64_t v) {
                v = csub(csub(v, q2), q);
                uint64_t r = mul_shoup(sub_mod(cx[e], v, q), f, fs, q);
                if (EPI == 2) r = add_mod(dst[e], r, q);
                dst[e] = r;
            });
    }
}

// inverse phase A: rows (lazy output < 2q; FP: signed lazy doubles in place)
template <int L1, bool FP>
__global__ void __launch_bounds__(kGroups * 32) k_rns_inv_rows(uint64_t* __restrict__ data, const RnsNttArgs a) {
    constexpr uint32_t ROW = 1u << kL2, ROWS = 1u << L1;
    extern __shared__ uint64_t sm[];
    const uint32_t tid = threadIdx.x;
    const uint32_t g = tid / 32, gt = tid % 32;
    const uint32_t rowblk = blockIdx.x % (ROWS / kGroups);
    const uint32_t limb_flat = blockIdx.x / (ROWS / kGroups);
    const uint32_t prime = a.limb_prime[limb_flat % a.limbs];
    const size_t N = size_t(1) << (L1 + kL2);
    const uint64_t* itw = a.itw + prime * N;
    const uint64_t* itws = a.itws + prime * N;
    const uint64_t q = a.q[prime];
    const uint32_t R = rowblk * kGroups + g;
    uint64_t* row = limb_ptr(data, a, limb_flat, L1 + kL2) + static_cast<size_t>(R) * ROW;
    const uint64_t* src = src_ptr(data, a, limb_flat, L1 + kL2) + static_cast<size_t>(R) * ROW;
    if constexpr (FP) {
        double* drow = reinterpret_cast<double*>(row);
        sub_inv_d<kL2>(
            reinterpret_cast<double*>(sm) + g * ROW, gt, a.itwd + prime * N, dmod_of(q),
            [&](uint32_t m) { return m * (ROWS + R); }, [&](uint32_t e) { return __ull2double_rn(src[e]); },
            [&](uint32_t e, double v, int) { drow[e] = v; });
    } else {
        sub_inv<kL2>(
            sm + g * ROW, gt, itw, itws, q, [&](uint32_t m) { return m * (ROWS + R); },
            [&](uint32_t e) { return src[e]; }, [&](uint32_t e, uint64_t v, int) { row[e] = v; });
    }
}

// inverse phase B: columns, n^-1 on the x-half of the last stage, full reduction
template <int L1, bool FP>
__global__ void __launch_bounds__(kGroups * (1 << L1) / 8) k_rns_inv_cols(uint64_t* __restrict__ data,
                                                                         const RnsNttArgs a) {
    constexpr uint32_t ROW = 1u << kL2;
    extern __shared__ uint64_t sm[];
    const uint32_t tid = threadIdx.x;
    const uint32_t g = tid % kGroups, gt = tid / kGroups;
    const uint32_t colblk = blockIdx.x % (ROW / kGroups);
    const uint32_t limb_flat = blockIdx.x / (ROW / kGroups);
    const uint32_t prime = a.limb_prime[limb_flat % a.limbs];
    const size_t N = size_t(1) << (L1 + kL2);
    const uint64_t* itw = a.itw + prime * N;
    const uint64_t* itws = a.itws + prime * N;
    const uint64_t q = a.q[prime];
    const uint64_t ninv = a.n_inv[prime], ninvs = a.n_inv_s[prime];
    const uint64_t sc = a.scale ? a.scale[limb_flat % a.limbs] : 0;
    const uint64_t scs = a.scale ? a.scale_s[limb_flat % a.limbs] : 0;
    uint64_t* poly = limb_ptr(data, a, limb_flat, L1 + kL2) + colblk * kGroups + g;
    if constexpr (FP) {
        const DMod md = dmod_of(q);
        const double ninv_d = static_cast<double>(ninv), sc_d = static_cast<double>(sc);
        const double* dpoly = reinterpret_cast<const double*>(poly);
        sub_inv_d<L1>(
            reinterpret_cast<double*>(sm) + g * col_stride<L1>(), gt, a.itwd + prime * N, md,
            [](uint32_t m) { return m; }, [&](uint32_t e) { return dpoly[e * ROW]; },
            [&](uint32_t e, double v, int j) {
                if (j < 4) v = dmulmod(v, ninv_d, md);  // x-half of the m = 1 stage
                if (sc) v = dmulmod(v, sc_d, md);
                poly[e * ROW] = dto_residue(v, md);
            });
        return;
    }
    sub_inv<L1>(
        sm + g * col_stride<L1>(), gt, itw, itws, q, [](uint32_t m) { return m; },
        [&](uint32_t e) { return poly[e * ROW]; },
        [&](uint32_t e, uint64_t v, int j) {
            v = csub(v, q);
            if (j < 4) v = mul_shoup(v, ninv, ninvs, q);  // x-half of the m = 1 stage
            if (sc) v = mul_shoup(v, sc, scs, q);
            poly[e * ROW] = v;
        });
}

// Row phases of the FP64 form with bulk copies: a CTA's 16 rows are 32 KB of one limb,
// contiguous in memory, so one thread moves them between global and shared memory with a
// single cp.async.bulk each way (completion on an mbarrier for the load, a bulk group for the
// store) instead of 8-byte loads and stores from every thread, which keep the load/store
// queues full (lg_throttle) at a fraction of HBM bandwidth.  Shared memory: the exchange
// buffer, the 32 KB staging block and the mbarrier.  A load whose wait expires sets bit 1 of
// *a.fault and the CTA finishes on whatever the staging block holds.
constexpr long long kBulkWaitLimit = 1ll << 31;  // SM clocks, about a second

__device__ __forceinline__ bool rows_bulk_load(double* stage, const void* src, uint64_t* bar, uint32_t* fault) {
    constexpr uint32_t bytes = kGroups * (1u << kL2) * sizeof(uint64_t);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
        mbar_arrive_expect_tx(bar, bytes);
        bulk_load(stage, src, bytes, bar);
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(bar, 0, kBulkWaitLimit);
    if (!ok && fault) atomicOr(fault, 1u);
    return ok;
}

__device__ __forceinline__ void rows_bulk_store(void* dst, const double* stage) {
    constexpr uint32_t bytes = kGroups * (1u << kL2) * sizeof(uint64_t);
    fence_proxy_async_smem();  // this thread's staging writes, before the copy engine reads them
    __syncthreads();
    if (threadIdx.x == 0) {
        bulk_store(dst, stage, bytes);
        bulk_store_commit_and_drain();
    }
}

template <int L1, int EPI>
__global__ void __launch_bounds__(kGroups * 32) k_rns_fwd_rows_bulk(uint64_t* __restrict__ data, const RnsNttArgs a) {
    constexpr uint32_t ROW = 1u << kL2, ROWS = 1u << L1;
    extern __shared__ __align__(16) uint64_t sm[];
    double* xsm = reinterpret_cast<double*>(sm);               // exchange [kGroups][ROW]
    double* stage = xsm + kGroups * ROW;                       // staging [kGroups][ROW]
    uint64_t* bar = sm + (EPI ? 3 : 2) * kGroups * ROW;  // after the staging blocks
    const uint32_t tid = threadIdx.x;
    const uint32_t g = tid / 32, gt = tid % 32;
    const uint32_t rowblk = blockIdx.x % (ROWS / kGroups);
    const uint32_t limb_flat = blockIdx.x / (ROWS / kGroups);
    const uint32_t prime = a.limb_prime[limb_flat % a.limbs];
    const size_t N = size_t(1) << (L1 + kL2);
    const uint64_t q = a.q[prime];
    const DMod md = dmod_of(q);
    const uint32_t R = rowblk * kGroups + g;
    uint64_t* blk = limb_ptr(data, a, limb_flat, L1 + kL2) + static_cast<size_t>(rowblk) * kGroups * ROW;
    rows_bulk_load(stage, blk, bar, a.fault);
    double* my = stage + g * ROW;
    uint64_t* myu = reinterpret_cast<uint64_t*>(my);
    const double* twd = a.twd + prime * N;
    if (EPI == 0) {
        sub_fwd_d<kL2>(
            xsm + g * ROW, gt, twd, md, [&](uint32_t m) { return m * (ROWS + R); }, [&](uint32_t e) { return my[e]; },
            [&](uint32_t e, double v) { myu[e] = dto_residue(v, md); });
        rows_bulk_store(blk, stage);
    } else {
        // the epilogue's cx block (and for EPI 2 the dst block, into the data stage once every
        // thread has read its inputs) stream in by bulk copies while the transform runs; the
        // results go out with one bulk store
        const uint32_t poly = limb_flat / a.limbs, limb = limb_flat % a.limbs;
        const size_t blk_off = (static_cast<size_t>(limb) << (L1 + kL2)) + static_cast<size_t>(rowblk) * kGroups * ROW;
        const uint64_t* cx_blk = a.epi_cx + poly * a.epi_cx_stride + blk_off;
        uint64_t* dst_blk = a.epi_dst + poly * a.epi_dst_stride + blk_off;
        uint64_t* cxs = reinterpret_cast<uint64_t*>(stage + kGroups * ROW);  // [kGroups][ROW]
        uint64_t* bar2 = bar + 1;
        constexpr uint32_t bytes = kGroups * ROW * sizeof(uint64_t);
        if (tid == 0) {
            mbar_init(bar2, 1);
            mbar_init_fence();
            mbar_arrive_expect_tx(bar2, EPI == 2 ? 2 * bytes : bytes);
            bulk_load(cxs, cx_blk, bytes, bar2);
        }
        const uint64_t f = a.epi_f[limb], fs = a.epi_fs[limb];
        uint64_t* my_cx = cxs + g * ROW;
        const uint64_t* my_dst = reinterpret_cast<const uint64_t*>(my);
        sub_fwd_d_hooked<kL2>(
            xsm + g * ROW, gt, twd, md, [&](uint32_t m) { return m * (ROWS + R); }, [&](uint32_t e) { return my[e]; },
            [&](uint32_t e, double dv) {
                const uint64_t v = dto_residue(dv, md);
                uint64_t r = mul_shoup(sub_mod(my_cx[e], v, q), f, fs, q);
                if (EPI == 2) r = add_mod(my_dst[e], r, q);
                my_cx[e] = r;
            },
            [&]() {
                if (EPI == 2 && tid == 0) {
                    fence_proxy_async_smem();  // the data stage was read by the generic proxy
                    bulk_load(stage, dst_blk, bytes, bar2);
                }
            },
            [&]() {
                if (!mbar_wait_bounded(bar2, 0, kBulkWaitLimit) && a.fault) atomicOr(a.fault, 1u);
            });
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            bulk_store(dst_blk, cxs, bytes);
            bulk_store_commit_and_drain();
        }
    }
}

template <int L1>
__global__ void __launch_bounds__(kGroups * 32) k_rns_inv_rows_bulk(uint64_t* __restrict__ data, const RnsNttArgs a) {
    constexpr uint32_t ROW = 1u << kL2, ROWS = 1u << L1;
    extern __shared__ __align__(16) uint64_t sm[];
    double* xsm = reinterpret_cast<double*>(sm);
    double* stage = xsm + kGroups * ROW;
    uint64_t* bar = sm + 2 * kGroups * ROW;
    const uint32_t tid = threadIdx.x;
    const uint32_t g = tid / 32, gt = tid % 32;
    const uint32_t rowblk = blockIdx.x % (ROWS / kGroups);
    const uint32_t limb_flat = blockIdx.x / (ROWS / kGroups);
    const uint32_t prime = a.limb_prime[limb_flat % a.limbs];
    const size_t N = size_t(1) << (L1 + kL2);
    const uint64_t q = a.q[prime];
    const uint32_t R = rowblk * kGroups + g;
    const size_t blk_off = static_cast<size_t>(rowblk) * kGroups * ROW;
    uint64_t* blk = limb_ptr(data, a, limb_flat, L1 + kL2) + blk_off;
    const uint64_t* src = src_ptr(data, a, limb_flat, L1 + kL2) + blk_off;
    rows_bulk_load(stage, src, bar, a.fault);
    double* my = stage + g * ROW;
    const uint64_t* myu = reinterpret_cast<const uint64_t*>(my);
    sub_inv_d<kL2>(
        xsm + g * ROW, gt, a.itwd + prime * N, dmod_of(q), [&](uint32_t m) { return m * (ROWS + R); },
        [&](uint32_t e) { return __ull2double_rn(myu[e]); }, [&](uint32_t e, double v, int) { my[e] = v; });
    rows_bulk_store(blk, stage);
}

// N = 2^10 .. 2^12: one CTA per limb polynomial, the register-blocked single-modulus transform
// of ntt_core.cuh with the limb's prime tables, plus the same slot maps, out-of-place input,
// inverse scaling and moddown epilogue as the 2-D kernels
template <int LOGN, int EPI>
__global__ void __launch_bounds__(NttPlan<LOGN>::T) k_rns_small_fwd(uint64_t* __restrict__ data, const RnsNttArgs a) {
    constexpr size_t N = size_t(1) << LOGN;
    __shared__ uint64_t sm[N];
    const uint32_t limb_flat = blockIdx.x;
    const uint32_t poly = limb_flat / a.limbs, limb = limb_flat % a.limbs;
    const uint32_t prime = a.limb_prime[limb];
    const uint64_t* tw = a.tw + prime * N;
    const uint64_t* tws = a.tws + prime * N;
    const uint64_t q = a.q[prime];
    uint64_t* dst = limb_ptr(data, a, limb_flat, LOGN);
    const uint64_t* src = src_ptr(data, a, limb_flat, LOGN);
    if (EPI == 0) {
        ntt_forward_cta<LOGN>(
            sm, threadIdx.x, tw, tws, q, [&](uint32_t i) { return src[i]; },
            [&](int, uint32_t i, uint64_t v) { dst[i] = v; });
    } else {
        const uint64_t* cx = a.epi_cx + poly * a.epi_cx_stride + (static_cast<size_t>(limb) << LOGN);
        uint64_t* out = a.epi_dst + poly * a.epi_dst_stride + (static_cast<size_t>(limb) << LOGN);
        const uint64_t f = a.epi_f[limb], fs = a.epi_fs[limb];
        ntt_forward_cta<LOGN>(
            sm, threadIdx.x, tw, tws, q, [&](uint32_t i) { return src[i]; },
            [&](int, uint32_t i, uint64_t v) {
                uint64_t r = mul_shoup(sub_mod(cx[i], v, q), f, fs, q);
                if (EPI == 2) r = add_mod(out[i], r, q);
                out[i] = r;
            });
    }
}

template <int LOGN>
__global__ void __launch_bounds__(NttPlan<LOGN>::T) k_rns_small_inv(uint64_t* __restrict__ data, const RnsNttArgs a) {
    constexpr size_t N = size_t(1) << LOGN;
    __shared__ uint64_t sm[N];
    const uint32_t limb_flat = blockIdx.x;
    const uint32_t limb = limb_flat % a.limbs;
    const uint32_t prime = a.limb_prime[limb];
    const uint64_t q = a.q[prime];
    const uint64_t sc = a.scale ? a.scale[limb] : 0, scs = a.scale ? a.scale_s[limb] : 0;
    uint64_t* dst = limb_ptr(data, a, limb_flat, LOGN);
    const uint64_t* src = src_ptr(data, a, limb_flat, LOGN);
    ntt_inverse_cta<LOGN>(
        sm, threadIdx.x, a.itw + prime * N, a.itws + prime * N, a.n_inv[prime], a.n_inv_s[prime], q,
        [&](int, uint32_t i) { return src[i]; },
        [&](uint32_t i, uint64_t v) { dst[i] = sc ? mul_shoup(v, sc, scs, q) : v; });
}

template <int LOGN>
static cudaError_t rns_small_launch(uint64_t* data, const RnsNttArgs& a, size_t limb_polys, bool inverse,
                                    cudaStream_t s) {
    if (limb_polys > 0x7fffffffu) return cudaErrorInvalidValue;
    const unsigned blocks = static_cast<unsigned>(limb_polys);
    if (inverse) k_rns_small_inv<LOGN><<<blocks, NttPlan<LOGN>::T, 0, s>>>(data, a);
    else if (a.epi == 0) k_rns_small_fwd<LOGN, 0><<<blocks, NttPlan<LOGN>::T, 0, s>>>(data, a);
    else if (a.epi == 1) k_rns_small_fwd<LOGN, 1><<<blocks, NttPlan<LOGN>::T, 0, s>>>(data, a);
    else k_rns_small_fwd<LOGN, 2><<<blocks, NttPlan<LOGN>::T, 0, s>>>(data, a);
    return cudaGetLastError();
}

template <int L1>
static cudaError_t rns_launch(uint64_t* data, const RnsNttArgs& a, size_t limb_polys, bool inverse, cudaStream_t s) {
    constexpr uint32_t ROW = 1u << kL2, ROWS = 1u << L1;
    constexpr size_t col_smem = kGroups * col_stride<L1>() * sizeof(uint64_t);
    constexpr size_t row_smem = kGroups * ROW * sizeof(uint64_t);
    static_assert(col_smem <= 227 * 1024 && row_smem <= 227 * 1024, "shared memory");
    static std::atomic<uint64_t> attr_set{0};  // opt-in above 48 KB, once per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!(attr_set.load() >> dev & 1)) {
        const void* fns[] = {reinterpret_cast<const void*>(k_rns_fwd_cols<L1, false>),
                             reinterpret_cast<const void*>(k_rns_inv_cols<L1, false>),
                             reinterpret_cast<const void*>(k_rns_fwd_cols<L1, true>),
                             reinterpret_cast<const void*>(k_rns_inv_cols<L1, true>)};
        for (const void* fn : fns) {
            cudaError_t e =
                cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(col_smem));
            if (e != cudaSuccess) return e;
        }
        attr_set.fetch_or(uint64_t(1) << dev);
    }
    const size_t col_blocks = limb_polys * (ROW / kGroups), row_blocks = limb_polys * (ROWS / kGroups);
    if (col_blocks > 0x7fffffffu || row_blocks > 0x7fffffffu) return cudaErrorInvalidValue;
    const uint32_t col_threads = kGroups * (1u << L1) / 8, row_threads = kGroups * 32;
    const unsigned cb = static_cast<unsigned>(col_blocks), rb = static_cast<unsigned>(row_blocks);
    if (a.twd && a.itwd) {
        // every prime of the chain is below 2^50: the FP64-pipe form; its row phases move each
        // CTA's 32 KB block with bulk copies when every block address is 16-byte aligned
        const auto a16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
        const bool bulk = a16(data) && (a.poly_stride & 1u) == 0 && (!a.in || (a16(a.in) && (a.in_poly_stride & 1u) == 0)) &&
                          (a.epi == 0 || (a16(a.epi_cx) && a16(a.epi_dst) && (a.epi_cx_stride & 1u) == 0 &&
                                          (a.epi_dst_stride & 1u) == 0));
        constexpr size_t bulk_smem = 2 * row_smem + 16, bulk_epi_smem = 3 * row_smem + 16;
        static std::atomic<uint64_t> bulk_attr{0};
        if (bulk && !(bulk_attr.load() >> dev & 1)) {
            const void* fns[] = {reinterpret_cast<const void*>(k_rns_fwd_rows_bulk<L1, 0>),
                                 reinterpret_cast<const void*>(k_rns_fwd_rows_bulk<L1, 1>),
                                 reinterpret_cast<const void*>(k_rns_fwd_rows_bulk<L1, 2>),
                                 reinterpret_cast<const void*>(k_rns_inv_rows_bulk<L1>)};
            for (const void* fn : fns) {
                cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     static_cast<int>(bulk_epi_smem));
                if (e != cudaSuccess) return e;
            }
            bulk_attr.fetch_or(uint64_t(1) << dev);
        }
        if (!inverse) {
            k_rns_fwd_cols<L1, true><<<cb, col_threads, col_smem, s>>>(data, a);
            if (bulk) {
                if (a.epi == 0) k_rns_fwd_rows_bulk<L1, 0><<<rb, row_threads, bulk_smem, s>>>(data, a);
                else if (a.epi == 1) k_rns_fwd_rows_bulk<L1, 1><<<rb, row_threads, bulk_epi_smem, s>>>(data, a);
                else k_rns_fwd_rows_bulk<L1, 2><<<rb, row_threads, bulk_epi_smem, s>>>(data, a);
            } else if (a.epi == 0) k_rns_fwd_rows<L1, 0, true><<<rb, row_threads, row_smem, s>>>(data, a);
            else if (a.epi == 1) k_rns_fwd_rows<L1, 1, true><<<rb, row_threads, row_smem, s>>>(data, a);
            else k_rns_fwd_rows<L1, 2, true><<<rb, row_threads, row_smem, s>>>(data, a);
        } else {
            if (bulk) k_rns_inv_rows_bulk<L1><<<rb, row_threads, bulk_smem, s>>>(data, a);
            else k_rns_inv_rows<L1, true><<<rb, row_threads, row_smem, s>>>(data, a);
            k_rns_inv_cols<L1, true><<<cb, col_threads, col_smem, s>>>(data, a);
        }
        return cudaGetLastError();
    }
    if (!inverse) {
        k_rns_fwd_cols<L1, false><<<cb, col_threads, col_smem, s>>>(data, a);
        if (a.epi == 0) k_rns_fwd_rows<L1, 0, false><<<rb, row_threads, row_smem, s>>>(data, a);
        else if (a.epi == 1) k_rns_fwd_rows<L1, 1, false><<<rb, row_threads, row_smem, s>>>(data, a);
        else k_rns_fwd_rows<L1, 2, false><<<rb, row_threads, row_smem, s>>>(data, a);
    } else {
        k_rns_inv_rows<L1, false><<<rb, row_threads, row_smem, s>>>(data, a);
        k_rns_inv_cols<L1, false><<<cb, col_threads, col_smem, s>>>(data, a);
    }
    return cudaGetLastError();
}

cudaError_t rns_ntt(uint64_t* data, const RnsNttArgs& a, uint32_t log_n, size_t polys, bool inverse, cudaStream_t s) {
    const size_t limb_polys = polys * a.limbs;
    if (limb_polys == 0) return cudaSuccess;
    switch (log_n) {
        case 10: return rns_small_launch<10>(data, a, limb_polys, inverse, s);
        case 11: return rns_small_launch<11>(data, a, limb_polys, inverse, s);
        case 12: return rns_small_launch<12>(data, a, limb_polys, inverse, s);
        case 13: return rns_launch<5>(data, a, limb_polys, inverse, s);
        case 14: return rns_launch<6>(data, a, limb_polys, inverse, s);
        case 15: return rns_launch<7>(data, a, limb_polys, inverse, s);
        case 16: return rns_launch<8>(data, a, limb_polys, inverse, s);
        case 17: return rns_launch<9>(data, a, limb_polys, inverse, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cbs
