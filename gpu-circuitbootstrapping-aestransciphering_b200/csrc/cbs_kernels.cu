// cbs_kernels.cu -- fused circuit-bootstrapping kernels for sm_100a.
//
// k_blind_rotate: one CTA per LWE ciphertext runs the whole GINX blind rotation of the
//   reference's batch path (bitwise/src/cirbts/cirbts-batch.cu:3293-4629 with the kernels
//   of bitwise/src/cirbts/kernel.cu:473-559 and :3008-3055) without leaving the SM: the
//   accumulator stays in shared memory for all n steps; per step each gadget digit is
//   computed on the fly while it is loaded into the NTT, the NTT output stays in
//   registers and is multiplied against the bootstrapping key with 128-bit lazy
//   accumulation (one Barrett reduction per output), the two products are inverse
//   transformed and rotate-added (acc += X^a * t - t) in the coefficient domain.  It then
//   finalizes (cirbts-batch.cu:2622-2642) and emits the multi-value split
//   ct_j = acc * X^-j (kernel.cu:7498-7536) in the NTT domain.
// k_trace_ss: one CTA per MV RLWE runs all HomTrace rounds and the SchemeSwitch
//   (cirbts-batch.cu:1656-1789; kernel.cu:7832-7888, :8407-8446) with the ciphertext
//   resident in shared memory, writing both RGSW rows (kernel.cu:7776-7789 layout).
// k_cmux_level: one CTA per CMux of a LUT tree level (examples/aes_transcipher/
//   gpu_lut.cuh:521-595): delta, INTT, gadget digits, NTT, MAC against the RGSW control,
//   add ct0.
#include "cbs_kernels.cuh"
#include "common.cuh"
#include "ntt_core.cuh"

namespace cbs {

__device__ __forceinline__ uint64_t reduce128(u128 x, const RingTables& t) {
    return csub(barrett_reduce_128(x, t.q, t.ratio0, t.ratio1), t.q);
}

// gadget digit d of x (least significant first), returned in [0, q)
__device__ __forceinline__ uint64_t digit_mod(uint64_t x, const Gadget& g, uint32_t d) {
    int64_t v = gadget_prepare(x, g);
    int32_t r = 0;
    for (uint32_t i = 0; i <= d; ++i) r = peel_digit(v, g.gbits);
    return signed_to_mod(r, g.q);
}

// acc += X^{e} t - t (coefficient domain)
template <uint32_t N, uint32_t T>
__device__ __forceinline__ void rotate_add(uint64_t* acc, const uint64_t* t, uint32_t e, uint32_t tid, uint64_t q) {
#pragma unroll
    for (uint32_t k = 0; k < N / T; ++k) {
        const uint32_t i = tid + k * T;
        const uint32_t s = (i + 2 * N - e) & (2 * N - 1);
        uint64_t v = (s < N) ? t[s] : t[s - N];
        if (s >= N) v = v ? q - v : 0;
        acc[i] = add_mod(acc[i], sub_mod(v, t[i], q), q);
    }
}

template <int LOGN>
__global__ void __launch_bounds__(NttPlan<LOGN>::T, 256 / NttPlan<LOGN>::T + (NttPlan<LOGN>::T < 512))
    k_blind_rotate(const BlindRotateArgs a) {
    constexpr uint32_t N = 1u << LOGN, T = NttPlan<LOGN>::T, TWO_N = 2 * N;
    extern __shared__ uint64_t smem[];
    uint64_t* acc0 = smem;
    uint64_t* acc1 = smem + N;
    uint64_t* scr = smem + 2 * N;
    uint64_t* tb = smem + 3 * N;
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const RingTables& t = a.t;
    const uint64_t Q = t.q;

    // acc = (0, X^{-b~} * TV)   (kernel.cu:7328-7358)
    {
        const uint32_t bt = special_ms_f(a.b[ct], TWO_N, a.q_lwe, a.bitwidth);
        for (uint32_t i = tid; i < N; i += T) {
            acc0[i] = 0;
            acc1[i] = rot_neg<N>(a.tv, bt, i, Q);
        }
    }
    __syncthreads();

    const uint32_t l2 = 2 * a.digits;
    const uint64_t* arow = a.a + static_cast<size_t>(ct) * a.a_stride;
    for (uint32_t step = 0; step < a.n; ++step) {
        const uint32_t at = special_ms_f(__ldg(arow + step), TWO_N, a.q_lwe, a.bitwidth);
        const uint64_t* ek = a.bsk + static_cast<size_t>(step) * l2 * 2 * N;
        uint64_t s0[8], s1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) s0[j] = s1[j] = 0;
        for (uint32_t r = 0; r < l2; ++r) {
            const uint64_t* src = (r & 1) ? acc1 : acc0;
            const uint32_t d = r >> 1;
            uint64_t x[8];
            ntt_forward_to_regs<LOGN>(
                scr, tid, t.rp, t.rps, Q, [&](uint32_t i) { return digit_mod(src[i], a.g, d); }, x);
            const ulonglong2* k0 = reinterpret_cast<const ulonglong2*>(ek + static_cast<size_t>(r) * 2 * N + 8 * tid);
            const ulonglong2* k1 =
                reinterpret_cast<const ulonglong2*>(ek + static_cast<size_t>(r) * 2 * N + N + 8 * tid);
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const ulonglong2 v0 = __ldg(k0 + h), v1 = __ldg(k1 + h);
                s0[2 * h] += mont_mul_lazy(x[2 * h], v0.x, Q, t.qneg_inv);
                s0[2 * h + 1] += mont_mul_lazy(x[2 * h + 1], v0.y, Q, t.qneg_inv);
                s1[2 * h] += mont_mul_lazy(x[2 * h], v1.x, Q, t.qneg_inv);
                s1[2 * h + 1] += mont_mul_lazy(x[2 * h + 1], v1.y, Q, t.qneg_inv);
            }
            __syncthreads();
        }
        uint64_t o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = reduce64(s0[j], Q, t.one_s);
        ntt_inverse_from_regs<LOGN>(scr, tid, t.irp, t.irps, t.n_inv, t.n_inv_s, Q, o,
                                    [&](uint32_t i, uint64_t v) { tb[i] = v; });
        __syncthreads();
        rotate_add<N, T>(acc0, tb, at, tid, Q);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = reduce64(s1[j], Q, t.one_s);
        ntt_inverse_from_regs<LOGN>(scr, tid, t.irp, t.irps, t.n_inv, t.n_inv_s, Q, o,
                                    [&](uint32_t i, uint64_t v) { tb[i] = v; });
        __syncthreads();
        rotate_add<N, T>(acc1, tb, at, tid, Q);
        __syncthreads();
    }

    // finalize: x N^-1, c1[j] += (gpow[j] >> 1) N^-1
    for (uint32_t i = tid; i < N; i += T) {
        acc0[i] = mul_shoup(acc0[i], t.n_inv, t.n_inv_s, Q);
        uint64_t v = mul_shoup(acc1[i], t.n_inv, t.n_inv_s, Q);
        if (i < a.num_lut) v = add_mod(v, a.gadd[i], Q);
        acc1[i] = v;
    }
    __syncthreads();

    // MV split ct_j = acc * X^{-j}, emitted in the NTT domain
    for (uint32_t j = 0; j < a.num_lut; ++j) {
        for (uint32_t p = 0; p < 2; ++p) {
            const uint64_t* src = p ? acc1 : acc0;
            uint64_t* dst = a.mv_out + ((static_cast<size_t>(ct) * a.num_lut + j) * 2 + p) * N;
            ntt_forward_cta<LOGN>(
                scr, tid, t.rp, t.rps, Q, [&](uint32_t i) { return rot_neg<N>(src, j, i, Q); },
                [&](int, uint32_t i, uint64_t v) { dst[i] = v; });
            __syncthreads();
        }
    }
}

template <int LOGN>
__global__ void __launch_bounds__(NttPlan<LOGN>::T, 256 / NttPlan<LOGN>::T + (NttPlan<LOGN>::T < 512))
    k_trace_ss(const TraceArgs a) {
    constexpr uint32_t N = 1u << LOGN, T = NttPlan<LOGN>::T;
    extern __shared__ uint64_t smem[];
    uint64_t* c0 = smem;
    uint64_t* c1 = smem + N;
    uint64_t* scr = smem + 2 * N;
    uint64_t* tb = smem + 3 * N;
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const RingTables& t = a.t;
    const uint64_t Q = t.q;
    const uint64_t* in = a.mv + static_cast<size_t>(ct) * 2 * N;
    for (uint32_t i = tid; i < 2 * N; i += T) smem[i] = in[i];
    __syncthreads();

    for (uint32_t r = 0; r < a.rounds; ++r) {
        const uint32_t* map = a.maps + static_cast<size_t>(r) * N;
        // sigma(c0) in the coefficient domain: permute in the NTT domain, then INTT
        ntt_inverse_cta<LOGN>(
            scr, tid, t.irp, t.irps, t.n_inv, t.n_inv_s, Q, [&](int, uint32_t i) { return c0[__ldg(map + i)]; },
            [&](uint32_t i, uint64_t v) { tb[i] = v; });
        __syncthreads();
        uint64_t s0[8], s1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) s0[j] = s1[j] = 0;
        for (uint32_t d = 0; d < a.digits_ht; ++d) {
            uint64_t x[8];
            ntt_forward_to_regs<LOGN>(
                scr, tid, t.rp, t.rps, Q, [&](uint32_t i) { return digit_mod(tb[i], a.g_ht, d); }, x);
            const uint64_t* k0 = a.ht_key + (static_cast<size_t>(r) * a.digits_ht + d) * 2 * N + 8 * tid;
            const uint64_t* k1 = k0 + N;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                s0[j] += mont_mul_lazy(x[j], __ldg(k0 + j), Q, t.qneg_inv);
                s1[j] += mont_mul_lazy(x[j], __ldg(k1 + j), Q, t.qneg_inv);
            }
            __syncthreads();
        }
        uint64_t pc1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) pc1[j] = c1[__ldg(map + 8 * tid + j)];
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t sl = 8 * tid + j;
            c0[sl] = add_mod(c0[sl], reduce64(s0[j], Q, t.one_s), Q);
            c1[sl] = add_mod(add_mod(c1[sl], reduce64(s1[j], Q, t.one_s), Q), pc1[j], Q);
        }
        __syncthreads();
    }

    uint64_t* out = a.rgsw + static_cast<size_t>(ct) * 4 * N;
    for (uint32_t i = tid; i < 2 * N; i += T) out[2 * N + i] = smem[i];  // trace row (type 1)

    // SchemeSwitch: digits of INTT(c0) against the s^2 key; row type 0 = (c1 + ks0, ks1)
    ntt_inverse_cta<LOGN>(
        scr, tid, t.irp, t.irps, t.n_inv, t.n_inv_s, Q, [&](int, uint32_t i) { return c0[i]; },
        [&](uint32_t i, uint64_t v) { tb[i] = v; });
    __syncthreads();
    uint64_t s0[8], s1[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) s0[j] = s1[j] = 0;
    for (uint32_t d = 0; d < a.digits_ss; ++d) {
        uint64_t x[8];
        ntt_forward_to_regs<LOGN>(
            scr, tid, t.rp, t.rps, Q, [&](uint32_t i) { return digit_mod(tb[i], a.g_ss, d); }, x);
        const uint64_t* k0 = a.ss_key + static_cast<size_t>(d) * 2 * N + 8 * tid;
        const uint64_t* k1 = k0 + N;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            s0[j] += mont_mul_lazy(x[j], __ldg(k0 + j), Q, t.qneg_inv);
            s1[j] += mont_mul_lazy(x[j], __ldg(k1 + j), Q, t.qneg_inv);
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t sl = 8 * tid + j;
        out[sl] = add_mod(c1[sl], reduce64(s0[j], Q, t.one_s), Q);
        out[N + sl] = reduce64(s1[j], Q, t.one_s);
    }
}

template <int LOGN>
__global__ void __launch_bounds__(NttPlan<LOGN>::T, 256 / NttPlan<LOGN>::T + (NttPlan<LOGN>::T < 512))
    k_cmux_level(const CmuxLevelArgs a) {
    constexpr uint32_t N = 1u << LOGN, T = NttPlan<LOGN>::T;
    (void)T;
    extern __shared__ uint64_t smem[];
    uint64_t* d0 = smem;
    uint64_t* d1 = smem + N;
    uint64_t* scr = smem + 2 * N;
    const uint32_t i = blockIdx.x, lut = blockIdx.y, tid = threadIdx.x;
    const RingTables& t = a.t;
    const uint64_t Q = t.q;
    const uint32_t set = a.lut_sel ? __ldg(a.lut_sel + lut) : lut;
    const uint64_t* in0 = a.in + set * a.in_lut_stride + static_cast<size_t>(2 * i) * 2 * N;
    const uint64_t* in1 = in0 + 2 * N;
    ntt_inverse_cta<LOGN>(
        scr, tid, t.irp, t.irps, t.n_inv, t.n_inv_s, Q, [&](int, uint32_t k) { return sub_mod(in1[k], in0[k], Q); },
        [&](uint32_t k, uint64_t v) { d0[k] = v; });
    __syncthreads();
    ntt_inverse_cta<LOGN>(
        scr, tid, t.irp, t.irps, t.n_inv, t.n_inv_s, Q,
        [&](int, uint32_t k) { return sub_mod(in1[N + k], in0[N + k], Q); },
        [&](uint32_t k, uint64_t v) { d1[k] = v; });
    __syncthreads();

    const uint32_t bit = __ldg(a.ctrl_bits + static_cast<size_t>(lut) * 8 + a.level);
    const uint64_t* G = a.rgsw_all + static_cast<size_t>(bit) * a.rgsw_stride;
    u128 s0[8], s1[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) s0[j] = s1[j] = u128{0, 0};
    for (uint32_t r = 0; r < 2 * a.digits; ++r) {
        const uint64_t* src = (r & 1) ? d1 : d0;
        const uint32_t d = r >> 1;
        uint64_t x[8];
        ntt_forward_to_regs<LOGN>(
            scr, tid, t.rp, t.rps, Q, [&](uint32_t k) { return digit_mod(src[k], a.g, d); }, x);
        const uint64_t* k0 = G + static_cast<size_t>(r) * 2 * N + 8 * tid;
        const uint64_t* k1 = k0 + N;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            add_wide(s0[j], mul_wide(x[j], __ldg(k0 + j)));
            add_wide(s1[j], mul_wide(x[j], __ldg(k1 + j)));
        }
        __syncthreads();
    }
    uint64_t* out = a.out + (static_cast<size_t>(lut) * (a.in_count / 2) + i) * 2 * N;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t sl = 8 * tid + j;
        out[sl] = add_mod(in0[sl], reduce128(s0[j], t), Q);
        out[N + sl] = add_mod(in0[N + sl], reduce128(s1[j], t), Q);
    }
}

// Opt a kernel into its dynamic shared memory once per process (outside any stream capture:
// the first launch of every kernel happens in an eager call).
template <class K>
static cudaError_t set_smem(K kernel, size_t bytes) {
    static size_t configured = 0;
    if (configured >= bytes) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e == cudaSuccess) configured = bytes;
    return e;
}

template <int LOGN>
static cudaError_t br_launch(const BlindRotateArgs& a, uint32_t batch, cudaStream_t s) {
    const size_t smem = 4ull * (1u << LOGN) * sizeof(uint64_t);
    cudaError_t e = set_smem(k_blind_rotate<LOGN>, smem);
    if (e != cudaSuccess) return e;
    k_blind_rotate<LOGN><<<batch, NttPlan<LOGN>::T, smem, s>>>(a);
    return cudaGetLastError();
}

template <int LOGN>
static cudaError_t trace_launch(const TraceArgs& a, uint32_t count, cudaStream_t s) {
    const size_t smem = 4ull * (1u << LOGN) * sizeof(uint64_t);
    cudaError_t e = set_smem(k_trace_ss<LOGN>, smem);
    if (e != cudaSuccess) return e;
    k_trace_ss<LOGN><<<count, NttPlan<LOGN>::T, smem, s>>>(a);
    return cudaGetLastError();
}

template <int LOGN>
static cudaError_t cmux_launch(const CmuxLevelArgs& a, uint32_t luts, cudaStream_t s) {
    const size_t smem = 3ull * (1u << LOGN) * sizeof(uint64_t);
    cudaError_t e = set_smem(k_cmux_level<LOGN>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.in_count / 2, luts);
    k_cmux_level<LOGN><<<grid, NttPlan<LOGN>::T, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_blind_rotate(const BlindRotateArgs& a, uint32_t N, uint32_t batch, cudaStream_t s) {
    if (batch == 0) return cudaSuccess;
    switch (N) {
        case 1024: return br_launch<10>(a, batch, s);
        case 2048: return br_launch<11>(a, batch, s);
        case 4096: return br_launch<12>(a, batch, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_trace_schemeswitch(const TraceArgs& a, uint32_t N, uint32_t count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    switch (N) {
        case 1024: return trace_launch<10>(a, count, s);
        case 2048: return trace_launch<11>(a, count, s);
        case 4096: return trace_launch<12>(a, count, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_cmux_level(const CmuxLevelArgs& a, uint32_t N, uint32_t luts, cudaStream_t s) {
    if (luts == 0 || a.in_count < 2) return cudaSuccess;
    switch (N) {
        case 1024: return cmux_launch<10>(a, luts, s);
        case 2048: return cmux_launch<11>(a, luts, s);
        case 4096: return cmux_launch<12>(a, luts, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cbs
