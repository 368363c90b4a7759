// cbs_fft.cu -- blind rotation with the FP64 FFT external product.
//
// Same accumulator algorithm as k_blind_rotate (GINX binary key, bitwise/src/cirbts/
// cirbts-batch.cu:3293-4629), with the external product computed the way the reference's
// gate bootstrap and its split-FFT CBS backend do (bitwise/src/fft.cu:3614-3755,
// bitwise/src/cirbts/cirbts-fft.cu:22-180): the signed gadget digits of the coefficient-
// domain accumulator are folded, twisted and FFT'd in FP64, multiplied against the FFT of
// the bootstrapping key, inverse-transformed, rounded back to integers and reduced mod Q,
// then rotate-added.  The key polynomials are uniform mod Q (~2^53 centered), so each
// product carries an FP64 rounding error of ~2^18-2^20 per coefficient; that error is noise
// on the accumulator (the bound is stated and checked against the exact product in the
// tests), not a change of the algorithm.  One CTA (N/8 threads) per ciphertext, the
// accumulator in shared memory for all n steps, the spectra of each step in registers.
#include <cmath>
#include <complex>
#include <thread>
#include <type_traits>
#include <vector>

#include "cbs_kernels.cuh"
#include "common.cuh"
#include "fft_core.cuh"
#include "fft_kernels.cuh"
#include "fft_ops.cuh"
#include "tmem.cuh"

namespace cbs {

// Two halves of M/8 threads per CTA: half h owns accumulator polynomial h.  Per step:
//  1. all threads decompose the accumulator (coefficient domain, shared memory) into packed
//     signed digit pairs (a_e, a_(e+M)) of every digit, stored once in shared memory;
//  2. half h forward-transforms digit d of polynomial h and multiplies the spectrum against
//     both key columns of key row 2d + h (keys stored in the order the threads consume them,
//     so each load is one coalesced 512-byte warp access), accumulating two output spectra;
//  3. the halves swap partial sums through shared memory (swizzled, conflict-free) so half h
//     holds the full spectrum of output h and inverse-transforms it into registers;
//  4. output h is staged in this half's FFT buffer and each thread updates the accumulator
//     positions it owns: acc_h[i] += t_h[i - a] (negacyclic wrap) - t_h[i].
template <int LOGN, bool WIDE>
__global__ void __launch_bounds__(BrFftCfg<LOGN>::T, BrFftCfg<LOGN>::MIN_BLOCKS)
    k_blind_rotate_fft(const BlindRotateArgs a, const FftKeyArgs f) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, T = 2 * TH, TWO_N = 2 * N;
    using Tb = FftTab<LOGM>;
    using DigT = typename DigitPair<WIDE>::T;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* acc = smem;                                           // [2][N]
    double2* fs = reinterpret_cast<double2*>(smem + 2 * N);         // [2][M]
    double2* tab = fs + 2 * M;                                      // FftTab<LOGM>
    DigT* dig = reinterpret_cast<DigT*>(tab + Tb::size());          // [2][digits][M] digit pairs
    const double2* tws = tab + Tb::twist_off();
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const uint32_t h = tid / TH, ht = tid % TH;
    int64_t* my_acc = reinterpret_cast<int64_t*>(acc) + h * N;
    double2* my_fs = fs + h * M;
    const uint64_t Q = a.t.q;
    const uint32_t digits = a.digits;
    const int gbits = a.g.gbits;
    int64_t offset = 0;
    for (uint32_t k = 0; k < digits; ++k) offset += static_cast<int64_t>(1) << (gbits * k + gbits - 1);
    const int ign = a.g.ign;
    const uint64_t qhalf = Q >> 1;
    // (x_centred + 2^(ign-1)) >> ign is the balanced rounding of gadget_prepare; adding the
    // digit offset before the shift folds both into one constant
    const uint64_t round_c = (ign ? (uint64_t(1) << (ign - 1)) : 0) + (static_cast<uint64_t>(offset) << ign);
    // During the steps the accumulator holds y = centre(x) + round_c (an int64 in [lo_b, hi_b),
    // centre(x) = x - Q for x >= Q/2 as in gadget_prepare), so the prepared digit word is y >> ign
    // and an update adds a centred residue and corrects once by +-Q.
    const int64_t hi_b = static_cast<int64_t>(round_c + qhalf), Qs = static_cast<int64_t>(Q), lo_b = hi_b - Qs;
    auto to_offset = [&](uint64_t x) {
        return static_cast<int64_t>(x + round_c) - (x >= qhalf ? Qs : 0);
    };

    for (uint32_t i = tid; i < Tb::size(); i += T) tab[i] = f.tab[i];
    {
        const uint32_t bt = special_ms_f(a.b[ct], TWO_N, a.q_lwe, a.bitwidth);
        int64_t* y = reinterpret_cast<int64_t*>(acc);
        for (uint32_t i = tid; i < N; i += T) {
            y[i] = to_offset(0);
            const uint32_t s = (i + bt) & (TWO_N - 1);
            const uint64_t v = (s < N) ? a.tv[s] : a.tv[s - N];
            y[N + i] = to_offset((s < N) ? v : (v ? Q - v : 0));
        }
    }
    __syncthreads();

    // barrier over the TH threads of this half (named barrier 1 + h; 0 is __syncthreads)
    auto half_bar = [h]() {
        if (h == 0) asm volatile("bar.sync 1, %0;" ::"n"(TH) : "memory");
        else asm volatile("bar.sync 2, %0;" ::"n"(TH) : "memory");
    };
    const uint32_t l2 = 2 * digits;
    const int32_t dbias = 1 << (gbits - 1);
    const uint64_t* arow = a.a + static_cast<size_t>(ct) * a.a_stride;
    for (uint32_t step = 0; step < a.n; ++step) {
        const uint32_t at = special_ms_f(__ldg(arow + step), TWO_N, a.q_lwe, a.bitwidth);
        // 1. digits of this half's polynomial.  Thread ht writes (and its first FFT pass
        //    reads) exactly the positions ht + j*TH it owns, so no barrier is needed for dig;
        //    the barrier after this loop orders the previous step's reads of my_fs before
        //    the first transform writes it.
        const uint32_t fmask = (1u << gbits) - 1u;
        for (uint32_t e = ht; e < M; e += TH) {
            const uint64_t wr = static_cast<uint64_t>(my_acc[e]) >> ign;
            const uint64_t wi = static_cast<uint64_t>(my_acc[e + M]) >> ign;
            DigT* dst = dig + h * digits * M + e;
            // biased digit fields (digit + 2^(gbits-1))
            for (uint32_t d = 0; d < digits; ++d)
                dst[d * M] = DigitPair<WIDE>::pack(static_cast<uint32_t>(wr >> (gbits * d)) & fmask,
                                                   static_cast<uint32_t>(wi >> (gbits * d)) & fmask);
        }
        half_bar();
        // 2. forward transforms and products
        const double2* ek = f.bskf + static_cast<size_t>(step) * l2 * 2 * M + ht;
        double2 y0[8], y1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) y0[j] = y1[j] = make_double2(0.0, 0.0);
        for (uint32_t d = 0; d < digits; ++d) {
            const DigT* dsrc = dig + (h * digits + d) * M;
            double2 x[8];
            fft_forward_to_regs<LOGM>(
                my_fs, ht, tab,
                [&](int j, uint32_t e) {
                    return cmul(DigitPair<WIDE>::unpack(dsrc[e], dbias), twist_at<LOGM>(tws, j, e));
                },
                x, half_bar);
            const double2* k0 = ek + static_cast<size_t>(2 * d + h) * 2 * M;  // key row 2d + h, slot-major
            const double2* k1 = k0 + M;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                cfma(y0[j], x[j], __ldg(k0 + j * TH));
                cfma(y1[j], x[j], __ldg(k1 + j * TH));
            }
            half_bar();  // the last pass's reads of my_fs are done before it is written again
        }
        // 3. swap partial sums: half 0 keeps output 0, half 1 keeps output 1
#pragma unroll
        for (int j = 0; j < 8; ++j) my_fs[cswz(8 * ht + j)] = h ? y0[j] : y1[j];
        __syncthreads();
        {
            const double2* take = fs + (1 - h) * M;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const double2 t = take[cswz(8 * ht + j)];
                y0[j] = cadd(h ? y1[j] : y0[j], t);
            }
        }
        __syncthreads();
        // 4. (X^a - 1) t_h in the frequency domain: slot s times psi_s^a - 1, then the inverse
        //    transform adds the rounded product into the accumulator positions this thread owns
        //    (the same positions its digit extraction reads: no barrier needed)
        {
            const uint32_t mb = mult_base<LOGN>(ht, at);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const double2 w = zeta_pow<LOGN>(tws, slot_exp<LOGN>(mb, at, j));
                y0[j] = cmul(y0[j], make_double2(w.x - 1.0, w.y));
            }
        }
        fft_inverse_from_regs<LOGM>(
            my_fs, ht, tab, y0,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                my_acc[e] = offset_add(my_acc[e], centred_residue(u.x * f.inv_m, f), lo_b, hi_b, Qs);
                my_acc[e + M] = offset_add(my_acc[e + M], centred_residue(u.y * f.inv_m, f), lo_b, hi_b, Qs);
            },
            half_bar);
    }
    __syncthreads();

    // finalize (cirbts-batch.cu:2622-2642) and the MV split ct_j = acc * X^-j in the
    // coefficient domain; the caller transforms mv_out to the NTT domain
    for (uint32_t i = tid; i < N; i += T) {
        // back from the offset form to [0, Q)
        const int64_t* y = reinterpret_cast<const int64_t*>(acc);
        const int64_t c0 = y[i] - static_cast<int64_t>(round_c), c1 = y[N + i] - static_cast<int64_t>(round_c);
        const uint64_t x0 = static_cast<uint64_t>(c0 < 0 ? c0 + Qs : c0);
        const uint64_t x1 = static_cast<uint64_t>(c1 < 0 ? c1 + Qs : c1);
        acc[i] = mul_shoup(x0, a.t.n_inv, a.t.n_inv_s, Q);
        uint64_t v = mul_shoup(x1, a.t.n_inv, a.t.n_inv_s, Q);
        if (i < a.num_lut) v = add_mod(v, a.gadd[i], Q);
        acc[N + i] = v;
    }
    __syncthreads();
    for (uint32_t j = 0; j < a.num_lut; ++j) {
        for (uint32_t p = 0; p < 2; ++p) {
            const uint64_t* src = acc + p * N;
            uint64_t* dst = a.mv_out + ((static_cast<size_t>(ct) * a.num_lut + j) * 2 + p) * N;
            for (uint32_t i = tid; i < N; i += T) {
                const uint32_t s = i + j;
                dst[i] = (s < N) ? src[s] : (src[s - N] ? Q - src[s - N] : 0);
            }
        }
    }
}

// Multi-bit blind rotation (the reference's CIRBTS_PBS_MULTIBIT = MB path: key grouping
// bitwise/src/cirbts/cirbts-init.cu:376-530, MB3 MAC kernel.cu:4585-4771) with FFT products.
// For binary s_i, prod_{i in G} (1 + (X^{a_i} - 1) s_i) = X^{sum a_i s_i}, so one step per
// group G of MB coefficients adds sum_S m_S (acc (x) K_S), K_S = RGSW(prod_{i in S} s_i),
// m_S = prod_{i in S} c_i, c_i = X^{a_i} - 1.  The external product is linear in the key,
// so per spectrum slot the combined key sum_S m_S(psi) K_S is formed in registers (Horner in
// the c_i: 2^MB - 1 complex multiply-adds) and multiplied once against the digit spectrum:
// the digit split, the 6 forward and 2 inverse transforms run once per group instead of
// once per coefficient, and the rotation needs no separate pass.  c_i(psi_s) comes from one
// twist-table lookup per group (zeta^(a_i e_t)) times an 8th root of unity per slot.
// Keys: [groups][keys][2*digits][2][N/2] spectra, subsets in the order {0} {1} {2}
// {0,1} {0,2} {1,2} {0,1,2} (MB = 3) or {0} {1} {0,1} (MB = 2).  MB = 4 is the reference's
// staged grouping (cirbts-init.cu:536-565 keys, cirbts-batch.cu:2767-2923 sequence): 8 keys
// {0} {1} {2} {3} {0,1} {0,2} {1,2} {0,1,2} per group of 4, applied as the MB = 3 step of
// coefficients 0-2 and then a one-bit step of coefficient 3 on a fresh digit split.
template <int MB>
__device__ __forceinline__ double2 mb_combined_key(const double2* kp, size_t kstride, const double2 (&c)[MB]) {
    if constexpr (MB == 2) {
        // c0 (K0 + c1 K01) + c1 K1
        double2 t = __ldg(kp);
        cfma(t, c[1], __ldg(kp + 2 * kstride));
        double2 r = cmul(c[0], t);
        cfma(r, c[1], __ldg(kp + kstride));
        return r;
    } else {
        // c0 (K0 + c1 (K01 + c2 K012) + c2 K02) + c1 (K1 + c2 K12) + c2 K2
        double2 t = __ldg(kp + 3 * kstride);
        cfma(t, c[2], __ldg(kp + 6 * kstride));
        double2 t2 = __ldg(kp);
        cfma(t2, c[1], t);
        cfma(t2, c[2], __ldg(kp + 4 * kstride));
        double2 u = __ldg(kp + kstride);
        cfma(u, c[2], __ldg(kp + 5 * kstride));
        double2 r = cmul(c[0], t2);
        cfma(r, c[1], u);
        cfma(r, c[2], __ldg(kp + 2 * kstride));
        return r;
    }
}

// Residency: the combined-key products keep many key loads in flight.  For MB = 2 one CTA per
// SM with the whole register file (no spills) is faster than two spilling CTAs (35.9 vs 40.5 us
// per bootstrap at N = 2048, n = 630); MB = 3 needs the warps of two CTAs to cover its seven
// key streams (58 vs 97 us).
template <int LOGN, int MB>
struct BrFftMbCfg {
    static constexpr int MIN_BLOCKS = 1;
};

template <int LOGN, int MB, bool WIDE>
__global__ void __launch_bounds__(BrFftCfg<LOGN>::T, BrFftMbCfg<LOGN, MB>::MIN_BLOCKS)
    k_blind_rotate_fft_mb(const BlindRotateArgs a, const FftKeyArgs f) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, T = 2 * TH, TWO_N = 2 * N;
    constexpr uint32_t KS = mb_group_keys(MB);
    using Tb = FftTab<LOGM>;
    using DigT = typename DigitPair<WIDE>::T;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* acc = smem;                                           // [2][N]
    double2* fs = reinterpret_cast<double2*>(smem + 2 * N);         // [2][M]
    double2* tab = fs + 2 * M;                                      // FftTab<LOGM>
    DigT* dig = reinterpret_cast<DigT*>(tab + Tb::size());          // [2][digits][M] digit pairs
    double2* cbuf = reinterpret_cast<double2*>(dig + 2 * a.digits * M);  // [step coefs][8][T] c_i per slot
    const double2* tws = tab + Tb::twist_off();
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const uint32_t h = tid / TH, ht = tid % TH;
    int64_t* my_acc = reinterpret_cast<int64_t*>(acc) + h * N;
    double2* my_fs = fs + h * M;
    const uint64_t Q = a.t.q;
    const uint32_t digits = a.digits;
    const int gbits = a.g.gbits;
    int64_t offset = 0;
    for (uint32_t k = 0; k < digits; ++k) offset += static_cast<int64_t>(1) << (gbits * k + gbits - 1);
    const int ign = a.g.ign;
    const uint64_t qhalf = Q >> 1;
    const uint64_t round_c = (ign ? (uint64_t(1) << (ign - 1)) : 0) + (static_cast<uint64_t>(offset) << ign);
    const int64_t hi_b = static_cast<int64_t>(round_c + qhalf), Qs = static_cast<int64_t>(Q), lo_b = hi_b - Qs;
    auto to_offset = [&](uint64_t x) {
        return static_cast<int64_t>(x + round_c) - (x >= qhalf ? Qs : 0);
    };

    for (uint32_t i = tid; i < Tb::size(); i += T) tab[i] = f.tab[i];
    {
        const uint32_t bt = special_ms_f(a.b[ct], TWO_N, a.q_lwe, a.bitwidth);
        int64_t* y = reinterpret_cast<int64_t*>(acc);
        for (uint32_t i = tid; i < N; i += T) {
            y[i] = to_offset(0);
            const uint32_t s = (i + bt) & (TWO_N - 1);
            const uint64_t v = (s < N) ? a.tv[s] : a.tv[s - N];
            y[N + i] = to_offset((s < N) ? v : (v ? Q - v : 0));
        }
    }
    __syncthreads();

    auto half_bar = [h]() {
        if (h == 0) asm volatile("bar.sync 1, %0;" ::"n"(TH) : "memory");
        else asm volatile("bar.sync 2, %0;" ::"n"(TH) : "memory");
    };
    const uint32_t l2 = 2 * digits;
    const int32_t dbias = 1 << (gbits - 1);
    const uint64_t* arow = a.a + static_cast<size_t>(ct) * a.a_stride;
    const uint32_t groups = (a.n + MB - 1) / MB;
    const size_t kstride = static_cast<size_t>(l2) * 2 * M;  // spectra between subsets of a group
    // one step: SMB coefficients idx0 .. idx0 + SMB - 1 against the group's keys slot(s) for
    // the subsets s of mb_key_mask(SMB, s)
    auto step = [&](auto smb_tag, uint32_t idx0, const double2* gkey, auto slot) {
        constexpr int SMB = decltype(smb_tag)::value;
        constexpr uint32_t SKS = (1u << SMB) - 1u;
        // zeta^(a_i e_t) per coefficient of the step (a_i = 0 past n: c_i = 0)
        // c_i(psi_s) = zeta^(a_i e_t) omega8^((a_i rev3(j)) mod 8) - 1 for the thread's 8 slots,
        // kept in shared memory for the step (thread-private entries: no barrier); omega8^k is
        // +-tw[(k mod 4) M/8] of the first-pass table
#pragma unroll
        for (int i = 0; i < SMB; ++i) {
            const uint32_t idx = idx0 + i;
            const uint32_t at = idx < a.n ? special_ms_f(__ldg(arow + idx), TWO_N, a.q_lwe, a.bitwidth) : 0u;
            const double2 ub = zeta_pow<LOGN>(tws, mult_base<LOGN>(ht, at));
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t r3 = ((j & 1) << 2) | (j & 2) | ((j >> 2) & 1);
                const uint32_t k = (at * r3) & 7u;
                double2 w = tab[(k & 3u) * (M / 8)];
                if (k & 4u) w = make_double2(-w.x, -w.y);
                const double2 v = cmul(ub, w);
                cbuf[(i * 8 + j) * T + tid] = make_double2(v.x - 1.0, v.y);
            }
        }
        // 1. digits of this half's polynomial (thread-private positions, as in the one-bit form)
        const uint32_t fmask = (1u << gbits) - 1u;
        for (uint32_t e = ht; e < M; e += TH) {
            const uint64_t wr = static_cast<uint64_t>(my_acc[e]) >> ign;
            const uint64_t wi = static_cast<uint64_t>(my_acc[e + M]) >> ign;
            DigT* dst = dig + h * digits * M + e;
            for (uint32_t d = 0; d < digits; ++d)
                dst[d * M] = DigitPair<WIDE>::pack(static_cast<uint32_t>(wr >> (gbits * d)) & fmask,
                                                   static_cast<uint32_t>(wi >> (gbits * d)) & fmask);
        }
        half_bar();
        // 2. forward transforms; per slot the combined key of row 2d + h, both columns
        const double2* gk = gkey + ht;
        double2 y0[8], y1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) y0[j] = y1[j] = make_double2(0.0, 0.0);
        for (uint32_t d = 0; d < digits; ++d) {
            const DigT* dsrc = dig + (h * digits + d) * M;
            double2 x[8];
            fft_forward_to_regs<LOGM>(
                my_fs, ht, tab,
                [&](int j, uint32_t e) {
                    return cmul(DigitPair<WIDE>::unpack(dsrc[e], dbias), twist_at<LOGM>(tws, j, e));
                },
                x, half_bar);
            // combined keys of row 2d + h, both columns, all 8 slots: subset by subset, the 16
            // key spectra of one subset are loaded together (16 independent loads in flight)
            const double2* k0 = gk + static_cast<size_t>(2 * d + h) * 2 * M;
            double2 kc0[8], kc1[8];
#pragma unroll
            for (int s = 0; s < static_cast<int>(SKS); ++s) {
                double2 ka[8], kb[8];
                const double2* ks = k0 + static_cast<size_t>(slot(s)) * kstride;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    ka[j] = __ldg(ks + j * TH);
                    kb[j] = __ldg(ks + M + j * TH);
                }
                const uint32_t mask = mb_key_mask(SMB, s);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    double2 m = make_double2(1.0, 0.0);
                    bool first = true;
#pragma unroll
                    for (int i = 0; i < SMB; ++i)
                        if (mask & (1u << i)) {
                            const double2 c = cbuf[(i * 8 + j) * T + tid];
                            m = first ? c : cmul(m, c);
                            first = false;
                        }
                    if (s == 0) {
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
            half_bar();  // the last pass's reads of my_fs are done before it is written again
        }
        // 3. swap partial sums: half 0 keeps output 0, half 1 keeps output 1
#pragma unroll
        for (int j = 0; j < 8; ++j) my_fs[cswz(8 * ht + j)] = h ? y0[j] : y1[j];
        __syncthreads();
        {
            const double2* take = fs + (1 - h) * M;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const double2 t = take[cswz(8 * ht + j)];
                y0[j] = cadd(h ? y1[j] : y0[j], t);
            }
        }
        __syncthreads();
        // 4. inverse transform, rounding, accumulate (the monomials are already in the keys)
        fft_inverse_from_regs<LOGM>(
            my_fs, ht, tab, y0,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                my_acc[e] = offset_add(my_acc[e], centred_residue(u.x * f.inv_m, f), lo_b, hi_b, Qs);
                my_acc[e + M] = offset_add(my_acc[e + M], centred_residue(u.y * f.inv_m, f), lo_b, hi_b, Qs);
            },
            half_bar);
    };
    for (uint32_t g = 0; g < groups; ++g) {
        const double2* gk = f.bskf + static_cast<size_t>(g) * KS * kstride;
        if constexpr (MB == 4) {
            // the staged grouping: the mb = 3 step of coefficients 0-2 (keys 0 1 2 4 5 6 7), then a
            // one-bit step of coefficient 3 (key 3) on the updated accumulator
            step(std::integral_constant<int, 3>{}, 4 * g, gk, [](int s) { return s < 3 ? s : s + 1; });
            if (4 * g + 3 < a.n) step(std::integral_constant<int, 1>{}, 4 * g + 3, gk, [](int) { return 3; });
        } else {
            step(std::integral_constant<int, MB>{}, g * MB, gk, [](int s) { return s; });
        }
    }
    __syncthreads();

    // finalize (cirbts-batch.cu:2622-2642) and the MV split, as in the one-bit form
    for (uint32_t i = tid; i < N; i += T) {
        const int64_t* y = reinterpret_cast<const int64_t*>(acc);
        const int64_t c0 = y[i] - static_cast<int64_t>(round_c), c1 = y[N + i] - static_cast<int64_t>(round_c);
        const uint64_t x0 = static_cast<uint64_t>(c0 < 0 ? c0 + Qs : c0);
        const uint64_t x1 = static_cast<uint64_t>(c1 < 0 ? c1 + Qs : c1);
        acc[i] = mul_shoup(x0, a.t.n_inv, a.t.n_inv_s, Q);
        uint64_t v = mul_shoup(x1, a.t.n_inv, a.t.n_inv_s, Q);
        if (i < a.num_lut) v = add_mod(v, a.gadd[i], Q);
        acc[N + i] = v;
    }
    __syncthreads();
    for (uint32_t j = 0; j < a.num_lut; ++j) {
        for (uint32_t p = 0; p < 2; ++p) {
            const uint64_t* src = acc + p * N;
            uint64_t* dst = a.mv_out + ((static_cast<size_t>(ct) * a.num_lut + j) * 2 + p) * N;
            for (uint32_t i = tid; i < N; i += T) {
                const uint32_t s = i + j;
                dst[i] = (s < N) ? src[s] : (src[s - N] ? Q - src[s - N] : 0);
            }
        }
    }
}

// Two-digit form of the grouped blind rotation (the 2^18 x 2 gadget).  Each half transforms both
// digits of its polynomial in lockstep (fft_forward2_to_regs: interleaved butterflies, one set
// of barriers, an exchange buffer per digit), then, per digit and subset S, multiplies the digit
// spectrum by m_S(psi) and accumulates it against the subset's key spectra of row 2d + h:
// y_c += (x_d m_S) K_S[2d + h][c].  Same arithmetic count as forming the combined key first; the
// two live digit spectra take the registers the combined-key accumulators held.
template <int LOGN, int MB, bool WIDE>
__global__ void __launch_bounds__(BrFftCfg<LOGN>::T, 1)
    k_blind_rotate_fft_mb_d2(const BlindRotateArgs a, const FftKeyArgs f) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, T = 2 * TH, TWO_N = 2 * N;
    constexpr uint32_t KS = (1u << MB) - 1u;
    constexpr uint32_t DIGITS = 2;
    using Tb = FftTab<LOGM>;
    using DigT = typename DigitPair<WIDE>::T;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* acc = smem;                                           // [2][N]
    double2* fs = reinterpret_cast<double2*>(smem + 2 * N);         // [2 halves][2 digits][M]
    double2* tab = fs + 4 * M;                                      // FftTab<LOGM>
    DigT* dig = reinterpret_cast<DigT*>(tab + Tb::size());          // [2][2][M] digit pairs
    double2* cbuf = reinterpret_cast<double2*>(dig + 2 * DIGITS * M);  // [MB][8][T] c_i per slot
    const double2* tws = tab + Tb::twist_off();
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const uint32_t h = tid / TH, ht = tid % TH;
    int64_t* my_acc = reinterpret_cast<int64_t*>(acc) + h * N;
    double2* my_fs0 = fs + (2 * h) * M;
    double2* my_fs1 = my_fs0 + M;
    const uint64_t Q = a.t.q;
    const int gbits = a.g.gbits;
    int64_t offset = 0;
    for (uint32_t k = 0; k < DIGITS; ++k) offset += static_cast<int64_t>(1) << (gbits * k + gbits - 1);
    const int ign = a.g.ign;
    const uint64_t qhalf = Q >> 1;
    const uint64_t round_c = (ign ? (uint64_t(1) << (ign - 1)) : 0) + (static_cast<uint64_t>(offset) << ign);
    const int64_t hi_b = static_cast<int64_t>(round_c + qhalf), Qs = static_cast<int64_t>(Q), lo_b = hi_b - Qs;
    auto to_offset = [&](uint64_t x) {
        return static_cast<int64_t>(x + round_c) - (x >= qhalf ? Qs : 0);
    };

    for (uint32_t i = tid; i < Tb::size(); i += T) tab[i] = f.tab[i];
    {
        const uint32_t bt = special_ms_f(a.b[ct], TWO_N, a.q_lwe, a.bitwidth);
        int64_t* y = reinterpret_cast<int64_t*>(acc);
        for (uint32_t i = tid; i < N; i += T) {
            y[i] = to_offset(0);
            const uint32_t s = (i + bt) & (TWO_N - 1);
            const uint64_t v = (s < N) ? a.tv[s] : a.tv[s - N];
            y[N + i] = to_offset((s < N) ? v : (v ? Q - v : 0));
        }
    }
    __syncthreads();

    auto half_bar = [h]() {
        if (h == 0) asm volatile("bar.sync 1, %0;" ::"n"(TH) : "memory");
        else asm volatile("bar.sync 2, %0;" ::"n"(TH) : "memory");
    };
    constexpr uint32_t l2 = 2 * DIGITS;
    const int32_t dbias = 1 << (gbits - 1);
    const uint64_t* arow = a.a + static_cast<size_t>(ct) * a.a_stride;
    const uint32_t groups = (a.n + MB - 1) / MB;
    constexpr size_t kstride = static_cast<size_t>(l2) * 2 * M;  // spectra between subsets of a group
    const uint32_t fmask = (1u << gbits) - 1u;
    for (uint32_t g = 0; g < groups; ++g) {
        // c_i(psi_s) for the thread's 8 slots, as in k_blind_rotate_fft_mb
#pragma unroll
        for (int i = 0; i < MB; ++i) {
            const uint32_t idx = g * MB + i;
            const uint32_t at = idx < a.n ? special_ms_f(__ldg(arow + idx), TWO_N, a.q_lwe, a.bitwidth) : 0u;
            const double2 ub = zeta_pow<LOGN>(tws, mult_base<LOGN>(ht, at));
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t r3 = ((j & 1) << 2) | (j & 2) | ((j >> 2) & 1);
                const uint32_t k = (at * r3) & 7u;
                double2 w = tab[(k & 3u) * (M / 8)];
                if (k & 4u) w = make_double2(-w.x, -w.y);
                const double2 v = cmul(ub, w);
                cbuf[(i * 8 + j) * T + tid] = make_double2(v.x - 1.0, v.y);
            }
        }
        // 1. both digits of this half's polynomial (thread-private positions)
        for (uint32_t e = ht; e < M; e += TH) {
            const uint64_t wr = static_cast<uint64_t>(my_acc[e]) >> ign;
            const uint64_t wi = static_cast<uint64_t>(my_acc[e + M]) >> ign;
            DigT* dst = dig + h * DIGITS * M + e;
#pragma unroll
            for (uint32_t d = 0; d < DIGITS; ++d)
                dst[d * M] = DigitPair<WIDE>::pack(static_cast<uint32_t>(wr >> (gbits * d)) & fmask,
                                                   static_cast<uint32_t>(wi >> (gbits * d)) & fmask);
        }
        half_bar();
        // 2. the two forward transforms in lockstep
        const DigT* d0 = dig + (h * DIGITS) * M;
        const DigT* d1 = d0 + M;
        double2 x0[8], x1[8];
        fft_forward2_to_regs<LOGM>(
            my_fs0, my_fs1, ht, tab,
            [&](int j, uint32_t e) { return cmul(DigitPair<WIDE>::unpack(d0[e], dbias), twist_at<LOGM>(tws, j, e)); },
            [&](int j, uint32_t e) { return cmul(DigitPair<WIDE>::unpack(d1[e], dbias), twist_at<LOGM>(tws, j, e)); },
            x0, x1, half_bar);
        // 3. products with the subsets' keys, row 2d + h, both columns
        const double2* gk = f.bskf + static_cast<size_t>(g) * KS * kstride + ht;
        double2 y0[8], y1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) y0[j] = y1[j] = make_double2(0.0, 0.0);
#pragma unroll
        for (uint32_t d = 0; d < DIGITS; ++d) {
            const double2* k0 = gk + static_cast<size_t>(2 * d + h) * 2 * M;
#pragma unroll
            for (int s = 0; s < static_cast<int>(KS); ++s) {
                double2 ka[8], kb[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    ka[j] = __ldg(k0 + s * kstride + j * TH);
                    kb[j] = __ldg(k0 + s * kstride + M + j * TH);
                }
                const uint32_t mask = mb_key_mask(MB, s);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    double2 t = d ? x1[j] : x0[j];
#pragma unroll
                    for (int i = 0; i < MB; ++i)
                        if (mask & (1u << i)) t = cmul(t, cbuf[(i * 8 + j) * T + tid]);
                    cfma(y0[j], t, ka[j]);
                    cfma(y1[j], t, kb[j]);
                }
            }
        }
        half_bar();  // the transforms' last reads of my_fs0 / my_fs1 are done before the swap writes
        // 4. swap partial sums: half 0 keeps output 0, half 1 keeps output 1
#pragma unroll
        for (int j = 0; j < 8; ++j) my_fs0[cswz(8 * ht + j)] = h ? y0[j] : y1[j];
        __syncthreads();
        {
            const double2* take = fs + (2 * (1 - h)) * M;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const double2 t = take[cswz(8 * ht + j)];
                y0[j] = cadd(h ? y1[j] : y0[j], t);
            }
        }
        __syncthreads();
        // 5. inverse transform, rounding, accumulate
        fft_inverse_from_regs<LOGM>(
            my_fs0, ht, tab, y0,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                my_acc[e] = offset_add(my_acc[e], centred_residue(u.x * f.inv_m, f), lo_b, hi_b, Qs);
                my_acc[e + M] = offset_add(my_acc[e + M], centred_residue(u.y * f.inv_m, f), lo_b, hi_b, Qs);
            },
            half_bar);
    }
    __syncthreads();

    // finalize and the MV split, as in the one-bit form
    for (uint32_t i = tid; i < N; i += T) {
        const int64_t* y = reinterpret_cast<const int64_t*>(acc);
        const int64_t c0 = y[i] - static_cast<int64_t>(round_c), c1 = y[N + i] - static_cast<int64_t>(round_c);
        const uint64_t x0 = static_cast<uint64_t>(c0 < 0 ? c0 + Qs : c0);
        const uint64_t x1 = static_cast<uint64_t>(c1 < 0 ? c1 + Qs : c1);
        acc[i] = mul_shoup(x0, a.t.n_inv, a.t.n_inv_s, Q);
        uint64_t v = mul_shoup(x1, a.t.n_inv, a.t.n_inv_s, Q);
        if (i < a.num_lut) v = add_mod(v, a.gadd[i], Q);
        acc[N + i] = v;
    }
    __syncthreads();
    for (uint32_t j = 0; j < a.num_lut; ++j) {
        for (uint32_t p = 0; p < 2; ++p) {
            const uint64_t* src = acc + p * N;
            uint64_t* dst = a.mv_out + ((static_cast<size_t>(ct) * a.num_lut + j) * 2 + p) * N;
            for (uint32_t i = tid; i < N; i += T) {
                const uint32_t s = i + j;
                dst[i] = (s < N) ? src[s] : (src[s - N] ? Q - src[s - N] : 0);
            }
        }
    }
}

// Paired form of the two-digit grouped blind rotation (mb = 2, 2^18 x 2 gadget): two
// ciphertexts per CTA of 512 threads, so an SM holds 16 warps instead of 8.  To fit 128
// registers and the shared memory of two ciphertexts, the work per group is split by output
// column instead of by input polynomial:
//  1. each half (128 threads) transforms the two digits of its polynomial in lockstep, with the
//     digits read straight from the accumulator (no digit buffer), and stores both spectra;
//  2. after a CTA barrier, the 512 threads split by output column, slot half and position: each
//     forms its 4 slots of output column mh for BOTH ciphertexts from all four digit spectra of
//     each, y_mh += x_row (sum_S m_S(psi) K_S[row][mh]) over the rows, so every key word loaded
//     feeds two ciphertexts; c_i(psi) = zeta^(a_i e_t) omega8^k - 1 is recomputed per slot;
//  3. after a second barrier (every spectrum read) the outputs go to the [mh][0] spectrum
//     buffers, and after a third, half h of each ciphertext inverse-transforms its column and
//     adds the rounded result into the accumulator positions it owns.
// The accumulator lives in tensor memory: a thread's transform reads and writes the same 16
// coefficients every group (positions e, e + M of its 8 slots), so they stay in its TMEM lane
// (ht, the same lane its warp quadrant reaches), 32 columns per half and ciphertext, 128 in all.
// Shared memory: the FFT tables once, then per ciphertext the spectra [2 halves][2 digits][N/2]
// (146 KB at N = 2048); the final accumulator passes through the spectra area for the MV
// split.  An odd batch's last CTA runs its second ciphertext as a copy of the first and writes
// nothing for it.
template <int LOGN, bool WIDE>
__global__ void __launch_bounds__(4 * ((1u << LOGN) / 16), 1)
    k_blind_rotate_fft_mb2_x2(const BlindRotateArgs a, const FftKeyArgs f, uint32_t batch) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, TWO_N = 2 * N;
    constexpr uint32_t KS = 3, DIGITS = 2, L2 = 2 * DIGITS;
    constexpr uint32_t TMEM_COLS = 128;  // 4 (ciphertext, half) pairs x 32 columns
    static_assert(TH == 128, "one TMEM lane per transform thread");
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    double2* tab = reinterpret_cast<double2*>(smem);                 // FftTab<LOGM>, shared
    const uint32_t tid = threadIdx.x, c2 = tid / (2 * TH), h = (tid / TH) & 1u, ht = tid % TH;
    const uint32_t lt = tid % (2 * TH);                               // thread within the ciphertext
    const uint32_t ct_raw = 2 * blockIdx.x + c2;
    const bool live = ct_raw < batch;
    const uint32_t ct = live ? ct_raw : batch - 1;
    // after the tables: the TMEM base address (16 bytes), then per ciphertext spec [2][2][M]
    constexpr size_t tab_words = (Tb::size() * sizeof(double2) + 15) / 16 * 2;  // 16-byte aligned, in u64
    constexpr size_t ct_words = 4 * M * 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + tab_words);
    double2* spec = reinterpret_cast<double2*>(smem + tab_words + 2 + c2 * ct_words);  // [p][d][M]
    const double2* tws = tab + Tb::twist_off();
    double2* my_s0 = spec + (2 * h) * M;
    double2* my_s1 = my_s0 + M;
    const uint64_t Q = a.t.q;
    const int gbits = a.g.gbits;
    int64_t offset = 0;
    for (uint32_t k = 0; k < DIGITS; ++k) offset += static_cast<int64_t>(1) << (gbits * k + gbits - 1);
    const int ign = a.g.ign;
    const uint64_t qhalf = Q >> 1;
    const uint64_t round_c = (ign ? (uint64_t(1) << (ign - 1)) : 0) + (static_cast<uint64_t>(offset) << ign);
    const int64_t hi_b = static_cast<int64_t>(round_c + qhalf), Qs = static_cast<int64_t>(Q), lo_b = hi_b - Qs;
    auto to_offset = [&](uint64_t x) {
        return static_cast<int64_t>(x + round_c) - (x >= qhalf ? Qs : 0);
    };

    if (tid < 32) tmem_alloc(tmem_slot, TMEM_COLS);
    for (uint32_t i = tid; i < Tb::size(); i += blockDim.x) tab[i] = f.tab[i];
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    // this thread's 32 columns: word 4j + {0, 1} = coefficient e_j (lo, hi), {2, 3} = e_j + M,
    // e_j = the transform's position of slot j; two 16-column halves (slots 0-3, 4-7)
    const uint32_t tacc = tmem_quadrant_addr(tmem_base, (2 * c2 + h) * 32);
    auto pack = [](uint32_t (&w)[16], int q, int64_t v) {
        w[q] = static_cast<uint32_t>(static_cast<uint64_t>(v));
        w[q + 1] = static_cast<uint32_t>(static_cast<uint64_t>(v) >> 32);
    };
    auto unpack = [](const uint32_t (&w)[16], int q) {
        return static_cast<int64_t>(static_cast<uint64_t>(w[q]) | (static_cast<uint64_t>(w[q + 1]) << 32));
    };
    {
        // polynomial 0 = 0, polynomial 1 = X^b times the test vector, in offset form
        const uint32_t bt = special_ms_f(a.b[ct], TWO_N, a.q_lwe, a.bitwidth);
        auto init = [&](uint32_t i) -> int64_t {
            if (h == 0) return to_offset(0);
            const uint32_t s = (i + bt) & (TWO_N - 1);
            const uint64_t v = (s < N) ? a.tv[s] : a.tv[s - N];
            return to_offset((s < N) ? v : (v ? Q - v : 0));
        };
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            uint32_t w[16];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                const uint32_t e = pass_index<LOGM, 3>(1u, ht, 4 * half + jj);
                pack(w, 4 * jj, init(e));
                pack(w, 4 * jj + 2, init(e + M));
            }
            tmem_store16(tacc + 16 * half, w);
        }
        tmem_wait_store();
    }
    __syncthreads();

    // named barriers: 1 + c2 over the ciphertext's 256 threads, 3 + 2 c2 + h over a half
    const uint32_t ct_bar = 1 + c2, half_id = 3 + 2 * c2 + h;
    auto ct_sync = [ct_bar]() { asm volatile("bar.sync %0, %1;" ::"r"(ct_bar), "n"(2 * TH) : "memory"); };
    auto half_bar = [half_id]() { asm volatile("bar.sync %0, %1;" ::"r"(half_id), "n"(TH) : "memory"); };
    const int32_t dbias = 1 << (gbits - 1);
    const uint32_t fmask = (1u << gbits) - 1u;
    const uint64_t* arow[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const uint32_t cr = 2 * blockIdx.x + c;
        arow[c] = a.a + static_cast<size_t>(cr < batch ? cr : batch - 1) * a.a_stride;
    }
    // the product phase's split of the 512 threads: output column mh, slot half sh, position mt
    const uint32_t mh = tid / (2 * TH), sh = (tid / TH) & 1u, mt = tid % TH;
    auto spec_of = [&](int c) {
        return reinterpret_cast<double2*>(smem + tab_words + 2 + c * ct_words);
    };
    const uint32_t groups = (a.n + 1) / 2;
    constexpr size_t kstride = static_cast<size_t>(L2) * 2 * M;  // spectra between subsets of a group
    // omega8 = tab[M/8] = (w8r, w8s w8r) and omega8^2 = tab[M/4] = (0, w8s)
    const double w8r = tab[M / 8].x, w8s = tab[2 * (M / 8)].y;
    for (uint32_t g = 0; g < groups; ++g) {
        // 1. the two digit transforms of polynomial h, digits read from the accumulator
        double2 x0[8], x1[8];
        {
            uint32_t wa[16], wb[16];
            tmem_load16(tacc, wa);
            tmem_load16(tacc + 16, wb);
            auto digit_pair = [&](int j, uint32_t e, int shift) {
                const uint32_t(&w)[16] = j < 4 ? wa : wb;
                const uint64_t wr = static_cast<uint64_t>(unpack(w, 4 * (j & 3))) >> (ign + shift);
                const uint64_t wi = static_cast<uint64_t>(unpack(w, 4 * (j & 3) + 2)) >> (ign + shift);
                return cmul(DigitPair<true>::unpack(make_uint2(static_cast<uint32_t>(wr) & fmask,
                                                               static_cast<uint32_t>(wi) & fmask),
                                                    dbias),
                            twist_at<LOGM>(tws, j, e));
            };
            fft_forward2_to_regs<LOGM>(
                my_s0, my_s1, ht, tab, [&](int j, uint32_t e) { return digit_pair(j, e, 0); },
                [&](int j, uint32_t e) { return digit_pair(j, e, gbits); }, x0, x1, half_bar);
        }
        half_bar();  // the transforms' last reads of my_s0 / my_s1 are done
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            my_s0[cswz(8 * ht + j)] = x0[j];
            my_s1[cswz(8 * ht + j)] = x1[j];
        }
        // the group's rotations of both ciphertexts (read before the barrier)
        const uint32_t idx0 = 2 * g, idx1 = idx0 + 1;
        uint32_t at[2][2];
        double2 ub[2][2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            at[c][0] = special_ms_f(__ldg(arow[c] + idx0), TWO_N, a.q_lwe, a.bitwidth);
            at[c][1] = idx1 < a.n ? special_ms_f(__ldg(arow[c] + idx1), TWO_N, a.q_lwe, a.bitwidth) : 0u;
            ub[c][0] = zeta_pow<LOGN>(tws, mult_base<LOGN>(mt, at[c][0]));
            ub[c][1] = zeta_pow<LOGN>(tws, mult_base<LOGN>(mt, at[c][1]));
        }
        __syncthreads();
        // 2. output column mh, slots 4 sh .. 4 sh + 3, of both ciphertexts: each key word feeds
        // both, through the combined key sum_S m_S(psi) K_S[row][mh] of each
        const double2* gk = f.bskf + static_cast<size_t>(g) * KS * kstride + static_cast<size_t>(mh) * M + mt;
        double2 y[2][4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const uint32_t j = 4 * sh + jj;
            const uint32_t r3 = ((j & 1) << 2) | (j & 2) | ((j >> 2) & 1);
            double2 cc[2][3];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    // omega8^k from its two distinct magnitudes (no table read)
                    const uint32_t k = (at[c][i] * r3) & 7u, k3 = k & 3u;
                    double2 w;
                    w.x = k3 == 0 ? 1.0 : (k3 == 2 ? 0.0 : (k3 == 1 ? w8r : -w8r));
                    w.y = k3 == 0 ? 0.0 : (k3 == 2 ? w8s : w8s * w8r);
                    if (k & 4u) w = make_double2(-w.x, -w.y);
                    cc[c][i] = cmul(ub[c][i], w);
                    cc[c][i].x -= 1.0;
                }
                cc[c][2] = cmul(cc[c][0], cc[c][1]);
                y[c][jj] = make_double2(0.0, 0.0);
            }
            const uint32_t xs = cswz(8 * mt + j);
#pragma unroll
            for (uint32_t row = 0; row < L2; ++row) {
                // row 2d + p: digit d of polynomial p, spectrum buffer [p][d]
                const double2* kr = gk + static_cast<size_t>(row) * 2 * M + j * TH;
                const double2 k0 = __ldg(kr), k1 = __ldg(kr + kstride), k2 = __ldg(kr + 2 * kstride);
                const uint32_t xo = ((row & 1u) * 2 + (row >> 1)) * M + xs;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    double2 kc = cmul(cc[c][0], k0);
                    cfma(kc, cc[c][1], k1);
                    cfma(kc, cc[c][2], k2);
                    cfma(y[c][jj], spec_of(c)[xo], kc);
                }
            }
        }
        __syncthreads();  // every spectrum read is done: the outputs take the [mh][0] buffers
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) spec_of(c)[(2 * mh) * M + cswz(8 * mt + 4 * sh + jj)] = y[c][jj];
        __syncthreads();
        double2 yv[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) yv[j] = my_s0[cswz(8 * ht + j)];
        half_bar();  // every output slot is in registers before the transform reuses the buffer
        // 3. inverse transform, rounding, accumulate into the TMEM accumulator (each 16-column
        // half read when its first slot arrives, written back after its last)
        uint32_t wacc[16];
        fft_inverse_from_regs<LOGM>(
            my_s0, ht, tab, yv,
            [&](int j, uint32_t e, double2 v) {
                if ((j & 3) == 0) tmem_load16(tacc + 16 * (j >> 2), wacc);
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                const int q = 4 * (j & 3);
                pack(wacc, q, offset_add(unpack(wacc, q), centred_residue(u.x * f.inv_m, f), lo_b, hi_b, Qs));
                pack(wacc, q + 2, offset_add(unpack(wacc, q + 2), centred_residue(u.y * f.inv_m, f), lo_b, hi_b, Qs));
                if ((j & 3) == 3) tmem_store16(tacc + 16 * (j >> 2), wacc);
            },
            half_bar);
        tmem_wait_store();
    }

    // the accumulator to shared memory ([2][N], natural order, in this ciphertext's spectra
    // area), then TMEM is released
    uint64_t* acc = reinterpret_cast<uint64_t*>(spec);
    ct_sync();  // the last inverse transforms' reads of the spectra area are done
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        uint32_t w[16];
        tmem_load16(tacc + 16 * half, w);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const uint32_t e = pass_index<LOGM, 3>(1u, ht, 4 * half + jj);
            acc[h * N + e] = static_cast<uint64_t>(unpack(w, 4 * jj));
            acc[h * N + e + M] = static_cast<uint64_t>(unpack(w, 4 * jj + 2));
        }
    }
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    if (tid < 32) tmem_dealloc(tmem_base, TMEM_COLS);

    // finalize and the MV split, as in the one-bit form
    for (uint32_t i = lt; i < N; i += 2 * TH) {
        const int64_t* y = reinterpret_cast<const int64_t*>(acc);
        const int64_t v0 = y[i] - static_cast<int64_t>(round_c), v1 = y[N + i] - static_cast<int64_t>(round_c);
        const uint64_t x0 = static_cast<uint64_t>(v0 < 0 ? v0 + Qs : v0);
        const uint64_t x1 = static_cast<uint64_t>(v1 < 0 ? v1 + Qs : v1);
        acc[i] = mul_shoup(x0, a.t.n_inv, a.t.n_inv_s, Q);
        uint64_t v = mul_shoup(x1, a.t.n_inv, a.t.n_inv_s, Q);
        if (i < a.num_lut) v = add_mod(v, a.gadd[i], Q);
        acc[N + i] = v;
    }
    ct_sync();
    if (!live) return;
    for (uint32_t j = 0; j < a.num_lut; ++j) {
        for (uint32_t p = 0; p < 2; ++p) {
            const uint64_t* src = acc + p * N;
            uint64_t* dst = a.mv_out + ((static_cast<size_t>(ct) * a.num_lut + j) * 2 + p) * N;
            for (uint32_t i = lt; i < N; i += 2 * TH) {
                const uint32_t s = i + j;
                dst[i] = (s < N) ? src[s] : (src[s - N] ? Q - src[s - N] : 0);
            }
        }
    }
}

cudaError_t ntt_forward(uint64_t* out, const uint64_t* in, const uint64_t* tw, const uint64_t* tws,
                        const cbs_dmodulus* mod, size_t dim, size_t batch, cudaStream_t s);

template <int LOGN, bool WIDE>
static cudaError_t br_fft_launch(const BlindRotateArgs& a, const FftKeyArgs& f, uint32_t batch, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    const size_t smem = 2ull * N * sizeof(uint64_t) + (2ull * M + FftTab<LOGN - 1>::size()) * sizeof(double2) +
                        2ull * a.digits * M * sizeof(typename DigitPair<WIDE>::T);
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    static size_t configured[64] = {};  // per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_blind_rotate_fft<LOGN, WIDE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_blind_rotate_fft<LOGN, WIDE><<<batch, BrFftCfg<LOGN>::T, smem, s>>>(a, f);
    return cudaGetLastError();
}

template <int LOGN>
static cudaError_t br_fft_launch(const BlindRotateArgs& a, const FftKeyArgs& f, uint32_t batch, cudaStream_t s) {
    return wide_digits(a.g.gbits) ? br_fft_launch<LOGN, true>(a, f, batch, s)
                                  : br_fft_launch<LOGN, false>(a, f, batch, s);
}

cudaError_t launch_blind_rotate_fft(const BlindRotateArgs& a, const FftKeyArgs& f, const cbs_dmodulus* d_mod,
                                    uint32_t N, uint32_t batch, cudaStream_t s, bool mv_ntt) {
    if (batch == 0) return cudaSuccess;
    if (a.g.gbits < 1 || a.g.gbits > 24 || a.digits < 1 || a.digits > 4) return cudaErrorInvalidValue;
    cudaError_t e;
    switch (N) {
        case 1024: e = br_fft_launch<10>(a, f, batch, s); break;
        case 2048: e = br_fft_launch<11>(a, f, batch, s); break;
        case 4096: e = br_fft_launch<12>(a, f, batch, s); break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess || !mv_ntt) return e;
    return ntt_forward(a.mv_out, a.mv_out, a.t.rp, a.t.rps, d_mod, N, static_cast<size_t>(batch) * a.num_lut * 2, s);
}

template <int LOGN, int MB, bool WIDE>
static cudaError_t br_fft_mb_launch(const BlindRotateArgs& a, const FftKeyArgs& f, uint32_t batch, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    const size_t smem = 2ull * N * sizeof(uint64_t) + (2ull * M + FftTab<LOGN - 1>::size()) * sizeof(double2) +
                        2ull * a.digits * M * sizeof(typename DigitPair<WIDE>::T) +
                        mb_step_coefs(MB) * 8ull * BrFftCfg<LOGN>::T * sizeof(double2);
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_blind_rotate_fft_mb<LOGN, MB, WIDE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_blind_rotate_fft_mb<LOGN, MB, WIDE><<<batch, BrFftCfg<LOGN>::T, smem, s>>>(a, f);
    return cudaGetLastError();
}

template <int LOGN, int MB, bool WIDE>
static cudaError_t br_fft_mb_d2_launch(const BlindRotateArgs& a, const FftKeyArgs& f, uint32_t batch,
                                       cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    const size_t smem = 2ull * N * sizeof(uint64_t) + (4ull * M + FftTab<LOGN - 1>::size()) * sizeof(double2) +
                        4ull * M * sizeof(typename DigitPair<WIDE>::T) + MB * 8ull * BrFftCfg<LOGN>::T * sizeof(double2);
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_blind_rotate_fft_mb_d2<LOGN, MB, WIDE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_blind_rotate_fft_mb_d2<LOGN, MB, WIDE><<<batch, BrFftCfg<LOGN>::T, smem, s>>>(a, f);
    return cudaGetLastError();
}

template <int LOGN>
static cudaError_t br_fft_mb2_x2_launch(const BlindRotateArgs& a, const FftKeyArgs& f, uint32_t batch,
                                        cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    constexpr size_t tab_bytes = (FftTab<LOGN - 1>::size() * sizeof(double2) + 15) / 16 * 16;
    const size_t smem = tab_bytes + 16 + 2 * (4ull * M * sizeof(double2));
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_blind_rotate_fft_mb2_x2<LOGN, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_blind_rotate_fft_mb2_x2<LOGN, true><<<(batch + 1) / 2, 4 * (N / 16), smem, s>>>(a, f, batch);
    return cudaGetLastError();
}

template <int LOGN, int MB>
static cudaError_t br_fft_mb_launch(const BlindRotateArgs& a, const FftKeyArgs& f, uint32_t batch, cudaStream_t s) {
    if constexpr (MB == 2 && LOGN == 11) {
        // two ciphertexts per CTA (digits read from the accumulator: any digit width up to 24
        // bits); also the default when no schedule was chosen or tuned (the fastest form on B200)
        if (a.digits == 2 && (a.schedule == CBS_BR_SCHEDULE_PAIRED || a.schedule == CBS_BR_SCHEDULE_AUTO))
            return br_fft_mb2_x2_launch<LOGN>(a, f, batch, s);
    }
    if constexpr (MB == 2) {
        // the two-digit gadget: both digit transforms in lockstep unless the digit-by-digit
        // schedule was chosen
        if (a.digits == 2 && a.schedule != CBS_BR_SCHEDULE_DIGITWISE)
            return wide_digits(a.g.gbits) ? br_fft_mb_d2_launch<LOGN, MB, true>(a, f, batch, s)
                                          : br_fft_mb_d2_launch<LOGN, MB, false>(a, f, batch, s);
    }
    return wide_digits(a.g.gbits) ? br_fft_mb_launch<LOGN, MB, true>(a, f, batch, s)
                                  : br_fft_mb_launch<LOGN, MB, false>(a, f, batch, s);
}

cudaError_t launch_blind_rotate_fft_mb(const BlindRotateArgs& a, const FftKeyArgs& f, const cbs_dmodulus* d_mod,
                                       uint32_t N, uint32_t batch, uint32_t mb, cudaStream_t s, bool mv_ntt) {
    if (batch == 0) return cudaSuccess;
    if (mb < 2 || mb > 4) return cudaErrorInvalidValue;  // N = 4096: the per-slot c_i exceed shared memory
    if (a.g.gbits < 1 || a.g.gbits > 24 || a.digits < 1 || a.digits > 4) return cudaErrorInvalidValue;
    cudaError_t e;
    switch (N) {
        case 1024:
            e = mb == 2 ? br_fft_mb_launch<10, 2>(a, f, batch, s)
                        : (mb == 3 ? br_fft_mb_launch<10, 3>(a, f, batch, s) : br_fft_mb_launch<10, 4>(a, f, batch, s));
            break;
        case 2048:
            e = mb == 2 ? br_fft_mb_launch<11, 2>(a, f, batch, s)
                        : (mb == 3 ? br_fft_mb_launch<11, 3>(a, f, batch, s) : br_fft_mb_launch<11, 4>(a, f, batch, s));
            break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess || !mv_ntt) return e;
    return ntt_forward(a.mv_out, a.mv_out, a.t.rp, a.t.rps, d_mod, N, static_cast<size_t>(batch) * a.num_lut * 2, s);
}

// ---- host side: FFT-domain key material ----

void host_dif(std::vector<cld>& a, const std::vector<cld>& w) {
    const size_t M = a.size();
    for (size_t h = M / 2; h >= 1; h /= 2) {
        const size_t stride = M / (2 * h);
        for (size_t s = 0; s < M; s += 2 * h)
            for (size_t j = 0; j < h; ++j) {
                const cld u = a[s + j], v = a[s + j + h];
                a[s + j] = u + v;
                a[s + j + h] = (u - v) * w[j * stride];
            }
        if (h == 1) break;
    }
}

template <int LOGM>
static void fft_tables_for(std::vector<double2>& tab) {
    using Tb = FftTab<LOGM>;
    constexpr uint32_t M = 1u << LOGM, N = 2 * M;
    using Pl = NttPlan<LOGM>;
    const long double pi = 3.141592653589793238462643383279502884L;
    auto tw = [&](uint32_t e) {
        const long double ang = 2.0L * pi * e / M;
        return make_double2(static_cast<double>(cosl(ang)), static_cast<double>(sinl(ang)));
    };
    tab.assign(Tb::size(), make_double2(0, 0));
    for (uint32_t e = 0; e < M / 2; ++e) tab[e] = tw(e);
    for (int p = 1; p < Pl::P; ++p) {
        const uint32_t m = Tb::pass_m(p), o = Tb::pass_off(p);
        const int r = Tb::pass_r(p);
        if (r == 3) {
            const uint32_t q = M / (8 * m);
            for (uint32_t j0 = 0; j0 < q; ++j0) {
                for (uint32_t k = 0; k < 4; ++k) tab[o + k * q + j0] = tw((j0 + k * q) * m);
                for (uint32_t k = 0; k < 2; ++k) tab[o + 4 * q + k * q + j0] = tw((j0 + k * q) * 2 * m);
                tab[o + 6 * q + j0] = tw(j0 * 4 * m);
            }
        } else if (r == 2) {
            const uint32_t q = M / (4 * m);
            for (uint32_t j0 = 0; j0 < q; ++j0) {
                tab[o + j0] = tw(j0 * m);
                tab[o + q + j0] = tw((j0 + q) * m);
                tab[o + 2 * q + j0] = tw(j0 * 2 * m);
            }
        } else {
            const uint32_t h = M / (2 * m);
            for (uint32_t j0 = 0; j0 < h; ++j0) tab[o + j0] = tw(j0 * m);
        }
    }
    for (uint32_t e = 0; e <= M / 2; ++e) {
        const long double ang = pi * e / N;
        tab[Tb::twist_off() + e] = make_double2(static_cast<double>(cosl(ang)), static_cast<double>(sinl(ang)));
    }
}

void fft_tables_host(uint32_t N, std::vector<double2>& tab) {
    switch (N) {
        case 1024: fft_tables_for<9>(tab); break;
        case 2048: fft_tables_for<10>(tab); break;
        case 4096: fft_tables_for<11>(tab); break;
        default: tab.clear();
    }
}

// NTT-domain key polynomials [count][N] (normal form, mod Q) -> FFT spectra.  Each key
// polynomial k (centred) yields one spectrum, or, when split_bits > 0 and polynomial index
// i % group == 0 (the first column of each key row), two: k_hi = round(k / 2^split_bits) and
// k_lo = k - k_hi 2^split_bits, so the output holds count + count / group spectra.  The
// halves keep products with small digits below 2^48, where the FP64 transform is exact after
// rounding.
void keys_to_fft_host(const host::NttTables& t, const uint64_t* keys_ntt, size_t count, std::vector<double2>& out,
                      uint32_t split_bits, uint32_t group) {
    const uint32_t N = t.n, M = N / 2;
    const uint64_t Q = t.q;
    const long double pi = 3.141592653589793238462643383279502884L;
    const bool split = split_bits > 0 && group > 0;
    std::vector<cld> w(M / 2), twist(M);
    for (uint32_t e = 0; e < M / 2; ++e) w[e] = std::polar(1.0L, 2.0L * pi * e / M);
    for (uint32_t e = 0; e < M; ++e) twist[e] = std::polar(1.0L, pi * e / N);
    // output spectrum index of input polynomial k (and k's lo half at +1 when split)
    auto out_index = [&](size_t k) { return split ? k + k / group + (k % group ? 1 : 0) : k; };
    const size_t total = split ? count + count / group : count;
    out.assign(total * M, make_double2(0, 0));
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th) {
        pool.emplace_back([&, th] {
            std::vector<uint64_t> c(N);
            std::vector<int64_t> v(N), hi(N), lo(N);
            std::vector<cld> z(M);
            // spectrum of the integer polynomial p, stored slot-major at spectrum index o:
            // slot s is consumed by thread s / 8 as its register j = s % 8, so it is stored at
            // j * (M / 8) + s / 8 and each warp load is contiguous
            auto emit = [&](const std::vector<int64_t>& p, size_t o) {
                for (uint32_t e = 0; e < M; ++e)
                    z[e] = cld(static_cast<long double>(p[e]), static_cast<long double>(p[e + M])) * twist[e];
                host_dif(z, w);
                for (uint32_t e = 0; e < M; ++e)
                    out[o * M + (e % 8) * (M / 8) + e / 8] =
                        make_double2(static_cast<double>(z[e].real()), static_cast<double>(z[e].imag()));
            };
            for (size_t k = th; k < count; k += nth) {
                std::copy(keys_ntt + k * N, keys_ntt + (k + 1) * N, c.begin());
                host::ntt_inverse_host(c.data(), t);
                for (uint32_t e = 0; e < N; ++e)
                    v[e] = c[e] > Q / 2 ? -static_cast<int64_t>(Q - c[e]) : static_cast<int64_t>(c[e]);
                const size_t o = out_index(k);
                if (split && k % group == 0) {
                    const int64_t half = int64_t(1) << (split_bits - 1);
                    for (uint32_t e = 0; e < N; ++e) {
                        hi[e] = (v[e] + half) >> split_bits;  // floor division: round to nearest
                        lo[e] = v[e] - hi[e] * (int64_t(1) << split_bits);
                    }
                    emit(hi, o);
                    emit(lo, o + 1);
                } else {
                    emit(v, o);
                }
            }
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace cbs
