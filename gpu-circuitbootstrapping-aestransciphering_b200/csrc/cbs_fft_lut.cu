// cbs_fft_lut.cu -- HomTrace + SchemeSwitch and the LUT-tree CMux with FP64 FFT products.
//
// Same algorithms as k_trace_ss and k_cmux_level (bitwise/src/cirbts/cirbts-batch.cu:
// 1656-1789, kernel.cu:7832-7888 and :8407-8446; examples/aes_transcipher/gpu_lut.cuh:
// 521-595), with the ciphertexts kept in the coefficient domain mod Q and every key product
// computed as a folded negacyclic FP64 FFT product (the external-product scheme of
// bitwise/src/fft.cu:3614-3755) rounded back mod Q:
//  * HomTrace round r: ct += KS_r(sigma_r(ct)) with sigma_r: X -> X^(N/2^r + 1) applied to
//    coefficients (a signed permutation), the balanced digits of sigma_r(a) transformed and
//    multiplied against the key spectra, two inverse transforms;
//  * SchemeSwitch: row type 0 = (b + KS(a)_0, KS(a)_1) against the s^2 key; row type 1 is the
//    trace output itself.  Both rows leave as FFT spectra, the form the CMux consumes;
//  * CMux: out = ct0 + RGSW (x) (ct1 - ct0), the eight digit spectra of the difference
//    multiplied against the row spectra, two inverse transforms, add ct0.
// The FP64 product error (~2^16-2^18 per coefficient at N = 2048 and a 54-bit Q) is noise,
// four orders of magnitude below the HomTrace noise the rows already carry.  One CTA of N/16
// threads per trace or CMux; the ciphertext stays in shared memory, spectra in registers.
#include "cbs_kernels.cuh"
#include "common.cuh"
#include "fft_core.cuh"
#include "fft_kernels.cuh"
#include "fft_ops.cuh"

namespace cbs {

template <int LOGN>
struct LutFftCfg {
    static constexpr uint32_t T = (1u << LOGN) / 16;  // one thread per 8 of the N/2 FFT points
    static constexpr int TRACE_BLOCKS = LOGN <= 10 ? 6 : (LOGN == 11 ? 3 : 1);
    static constexpr int CMUX_BLOCKS = LOGN <= 10 ? 8 : (LOGN == 11 ? 4 : 2);
};

// coefficient j of sigma(p) = p(X^k) for k^-1 = kinv (mod 2N): +p[i] or -p[i - N] with
// i = j kinv mod 2N
template <uint32_t N>
__device__ __forceinline__ uint64_t sigma_coeff(const uint64_t* p, uint32_t kinv, uint32_t j, uint64_t Q) {
    const uint32_t i = (j * kinv) & (2 * N - 1);
    const uint64_t v = p[i & (N - 1)];
    return (i < N || v == 0) ? v : Q - v;
}

// forward transform of the centred coefficient-domain polynomial p (mod Q) into x
template <int LOGM, class Bar>
__device__ __forceinline__ void fft_of_poly(double2* fs, uint32_t tid, const double2* tab, const uint64_t* p,
                                            uint64_t Q, double2 (&x)[8], Bar bar) {
    constexpr uint32_t M = 1u << LOGM;
    const double2* tws = tab + FftTab<LOGM>::twist_off();
    const uint64_t qhalf = Q >> 1;
    fft_forward_to_regs<LOGM>(
        fs, tid, tab,
        [&](int j, uint32_t e) {
            return cmul(make_double2(centred_double(p[e], Q, qhalf), centred_double(p[e + M], Q, qhalf)),
                        twist_at<LOGM>(tws, j, e));
        },
        x, bar);
}

// spectrum slot 8 tid + j of the forward transform is stored at j * (M/8) + tid (the order
// in which the consuming kernels' threads read it, one coalesced access per warp)
template <uint32_t T>
__device__ __forceinline__ void store_spectrum(double2* dst, uint32_t tid, const double2 (&x)[8]) {
#pragma unroll
    for (int j = 0; j < 8; ++j) dst[j * T + tid] = x[j];
}

// Key-switch products of one polynomial: for each gadget digit d, the forward transform of the
// balanced digit d of prep(e) (the prepared word of coefficient e) times the three key
// columns of row d ([k0_hi, k0_lo, k1] spectra, slot-major), accumulated into yh, yl, y1.
// The CTA barrier after each product orders the transform's last reads of fs before the next
// transform writes it; on return every prep() read of the CTA has completed.
template <int LOGM, class Prep>
__device__ __forceinline__ void key_switch_products(double2* fs, uint32_t tid, const double2* tab,
                                                    const double2* key, uint32_t digits, Prep prep, int gbits,
                                                    double2 (&yh)[8], double2 (&yl)[8], double2 (&y1)[8]) {
    constexpr uint32_t M = 1u << LOGM, T = M / 8;
    const double2* tws = tab + FftTab<LOGM>::twist_off();
#pragma unroll
    for (int j = 0; j < 8; ++j) yh[j] = yl[j] = y1[j] = make_double2(0.0, 0.0);
    for (uint32_t d = 0; d < digits; ++d) {
        double2 x[8];
        fft_forward_to_regs<LOGM>(
            fs, tid, tab,
            [&](int j, uint32_t e) {
                const int64_t wr = prep(e);
                const int64_t wi = prep(e + M);
                return cmul(make_double2(static_cast<double>(balanced_digit(wr, gbits, d)),
                                         static_cast<double>(balanced_digit(wi, gbits, d))),
                            twist_at<LOGM>(tws, j, e));
            },
            x, []() { __syncthreads(); });
        const double2* kh = key + static_cast<size_t>(d) * 3 * M + tid;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            cfma(yh[j], x[j], __ldg(kh + j * T));
            cfma(yl[j], x[j], __ldg(kh + M + j * T));
            cfma(y1[j], x[j], __ldg(kh + 2 * M + j * T));
        }
        __syncthreads();
    }
}

template <int LOGN>
__global__ void __launch_bounds__(LutFftCfg<LOGN>::T, LutFftCfg<LOGN>::TRACE_BLOCKS)
    k_trace_ss_fft(const TraceFftArgs a, const FftKeyArgs f) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, T = M / 8;
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* c0 = smem;                                     // [N] mask a
    uint64_t* c1 = smem + N;                                 // [N] body b
    double2* fs = reinterpret_cast<double2*>(smem + 2 * N);  // [M] transform exchange
    double2* tab = fs + M;                                   // FftTab<LOGM>
    const double2* tws = tab + Tb::twist_off();
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const uint64_t Q = a.g_ht.q;
    auto bar = []() { __syncthreads(); };

    for (uint32_t i = tid; i < Tb::size(); i += T) tab[i] = f.tab[i];
    {
        const uint64_t* in = a.mv + static_cast<size_t>(ct) * 2 * N;
        for (uint32_t i = tid; i < 2 * N; i += T) smem[i] = in[i];
    }
    __syncthreads();

    const int gb_ht = a.g_ht.gbits;
    for (uint32_t r = 0; r < a.rounds; ++r) {
        const uint32_t kinv = a.kinv[r];
        double2 yh[8], yl[8], y1[8];
        key_switch_products<LOGM>(fs, tid, tab, a.htf + static_cast<size_t>(r) * a.digits_ht * 3 * M, a.digits_ht,
                                  [&](uint32_t e) { return prepared_offset(sigma_coeff<N>(c0, kinv, e, Q), a.g_ht); },
                                  gb_ht, yh, yl, y1);
        // a += KS_0 = 2^S hi + lo (only this thread's positions; a's last reads were the digit
        // loads above, ordered by the barrier after the last product)
        fft_inverse_from_regs<LOGM>(
            fs, tid, tab, yh,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                c0[e] = add_mod(c0[e], mul_shoup(double_to_mod(u.x * f.inv_m, f, Q), a.split_pow, a.split_pow_s, Q), Q);
                c0[e + M] =
                    add_mod(c0[e + M], mul_shoup(double_to_mod(u.y * f.inv_m, f, Q), a.split_pow, a.split_pow_s, Q), Q);
            },
            bar);
        __syncthreads();
        fft_inverse_from_regs<LOGM>(
            fs, tid, tab, yl,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                c0[e] = add_mod(c0[e], double_to_mod(u.x * f.inv_m, f, Q), Q);
                c0[e + M] = add_mod(c0[e + M], double_to_mod(u.y * f.inv_m, f, Q), Q);
            },
            bar);
        __syncthreads();
        // sigma(b) at the positions this thread updates, read before any thread writes b (the
        // inverse transform below has CTA barriers between here and its stores)
        uint64_t sb_lo[8], sb_hi[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t e = tid + j * T;
            sb_lo[j] = sigma_coeff<N>(c1, kinv, e, Q);
            sb_hi[j] = sigma_coeff<N>(c1, kinv, e + M, Q);
        }
        // b += sigma(b) + KS_1
        fft_inverse_from_regs<LOGM>(
            fs, tid, tab, y1,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                c1[e] = add_mod(add_mod(c1[e], sb_lo[j], Q), double_to_mod(u.x * f.inv_m, f, Q), Q);
                c1[e + M] = add_mod(add_mod(c1[e + M], sb_hi[j], Q), double_to_mod(u.y * f.inv_m, f, Q), Q);
            },
            bar);
        __syncthreads();
    }

    double2* out = a.rgswf + static_cast<size_t>(ct) * 4 * M;
    {
        // row type 1: the trace output
        double2 x[8];
        fft_of_poly<LOGM>(fs, tid, tab, c0, Q, x, bar);
        store_spectrum<T>(out + 2 * M, tid, x);
        __syncthreads();
        fft_of_poly<LOGM>(fs, tid, tab, c1, Q, x, bar);
        store_spectrum<T>(out + 3 * M, tid, x);
        __syncthreads();
    }
    // SchemeSwitch: KS(a) against the s^2 key; row type 0 = (b + KS_0, KS_1), rebuilt in the
    // coefficient domain in place of (a, b)
    {
        double2 yh[8], yl[8], y1[8];
        key_switch_products<LOGM>(fs, tid, tab, a.ssf, a.digits_ss,
                                  [&](uint32_t e) { return prepared_offset(c0[e], a.g_ss); }, a.g_ss.gbits, yh, yl,
                                  y1);
        fft_inverse_from_regs<LOGM>(
            fs, tid, tab, yh,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                c0[e] = add_mod(c1[e], mul_shoup(double_to_mod(u.x * f.inv_m, f, Q), a.split_pow, a.split_pow_s, Q), Q);
                c0[e + M] =
                    add_mod(c1[e + M], mul_shoup(double_to_mod(u.y * f.inv_m, f, Q), a.split_pow, a.split_pow_s, Q), Q);
            },
            bar);
        __syncthreads();
        fft_inverse_from_regs<LOGM>(
            fs, tid, tab, yl,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                c0[e] = add_mod(c0[e], double_to_mod(u.x * f.inv_m, f, Q), Q);
                c0[e + M] = add_mod(c0[e + M], double_to_mod(u.y * f.inv_m, f, Q), Q);
            },
            bar);
        __syncthreads();
        fft_inverse_from_regs<LOGM>(
            fs, tid, tab, y1,
            [&](int j, uint32_t e, double2 v) {
                const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                c1[e] = double_to_mod(u.x * f.inv_m, f, Q);
                c1[e + M] = double_to_mod(u.y * f.inv_m, f, Q);
            },
            bar);
        __syncthreads();
    }
    double2 x[8];
    fft_of_poly<LOGM>(fs, tid, tab, c0, Q, x, bar);
    store_spectrum<T>(out, tid, x);
    __syncthreads();
    fft_of_poly<LOGM>(fs, tid, tab, c1, Q, x, bar);
    store_spectrum<T>(out + M, tid, x);
}

// prepared digit words (re, im) of component p of in1 - in0 into ws[M]
template <uint32_t N, uint32_t T>
__device__ __forceinline__ void cmux_diff_words(uint2* ws, const uint64_t* in0, const uint64_t* in1, uint32_t p,
                                                const DigitPrep& g, uint32_t tid) {
    constexpr uint32_t M = N / 2;
    for (uint32_t e = tid; e < M; e += T) {
        const uint32_t lo = p * N + e, hi = lo + M;
        const uint64_t dr = sub_mod(__ldg(in1 + lo), __ldg(in0 + lo), g.q);
        const uint64_t di = sub_mod(__ldg(in1 + hi), __ldg(in0 + hi), g.q);
        ws[e] = make_uint2(static_cast<uint32_t>(prepared_offset(dr, g)),
                           static_cast<uint32_t>(prepared_offset(di, g)));
    }
}

// forward transform of digit d of the prepared words src into x
template <int LOGM, class Bar>
__device__ __forceinline__ void cmux_digit_fft(double2* fs, uint32_t tid, const double2* tab, const uint2* src,
                                               int gbits, uint32_t d, double2 (&x)[8], Bar bar) {
    const double2* tws = tab + FftTab<LOGM>::twist_off();
    fft_forward_to_regs<LOGM>(
        fs, tid, tab,
        [&](int j, uint32_t e) {
            const uint2 w = src[e];
            return cmul(make_double2(static_cast<double>(balanced_digit(w.x, gbits, d)),
                                     static_cast<double>(balanced_digit(w.y, gbits, d))),
                        twist_at<LOGM>(tws, j, e));
        },
        x, bar);
}

// Digit spectra of the level-0 pair differences of fixed LUT tables, computed once: CTA
// (i, set, r) writes transform r = 2d + p of in[2i+1] - in[2i] (set `set`) to
// out[((set * pairs + i) * 2 digits + r) * M], slot-major as the CMux reads it.
template <int LOGN>
__global__ void __launch_bounds__(LutFftCfg<LOGN>::T) k_cmux_pair_spectra(const CmuxFftArgs a, const FftKeyArgs f,
                                                                            double2* out) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, T = M / 8;
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    uint2* ws = reinterpret_cast<uint2*>(smem);            // [M]
    double2* fs = reinterpret_cast<double2*>(ws + 2 * M);  // [M]
    double2* tab = fs + M;
    const uint32_t i = blockIdx.x, set = blockIdx.y, r = blockIdx.z, tid = threadIdx.x;
    for (uint32_t k = tid; k < Tb::size(); k += T) tab[k] = f.tab[k];
    const uint64_t* in0 = a.in + set * a.in_lut_stride + static_cast<size_t>(2 * i) * 2 * N;
    cmux_diff_words<N, T>(ws, in0, in0 + 2 * N, r & 1, a.g, tid);
    __syncthreads();
    double2 x[8];
    cmux_digit_fft<LOGM>(fs, tid, tab, ws, a.g.gbits, r >> 1, x, []() { __syncthreads(); });
    double2* dst = out + ((static_cast<size_t>(set) * gridDim.x + i) * gridDim.z + r) * M + tid;
#pragma unroll
    for (int j = 0; j < 8; ++j) dst[j * T] = x[j];
}

// One CMux of a LUT-tree level per CTA: ct0 = input 2i, ct1 = input 2i + 1 of the LUT's set,
// control = RGSW of bit ctrl_bits[lut][level].  The prepared digit words of both difference
// polynomials are computed once into shared memory (digits * gbits <= 32 bits per word);
// transform r = 2d + p takes digit d of polynomial p and multiplies it against row r.  With
// a.in_spec (level 0 over fixed tables) the digit spectra are read from k_cmux_pair_spectra's
// output instead (no decomposition, no forward transforms).  CTAs run pair-major within a
// LUT: the 128 CTAs of a LUT share its control's row spectra through L2, and the few tables
// of a round (4 x 16.7 MB of spectra at N = 2048) stay L2-resident across the LUTs.
template <int LOGN>
__global__ void __launch_bounds__(LutFftCfg<LOGN>::T, LutFftCfg<LOGN>::CMUX_BLOCKS)
    k_cmux_level_fft(const CmuxFftArgs a, const FftKeyArgs f) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, T = M / 8;
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    uint2* ws = reinterpret_cast<uint2*>(smem);         // [2][M] (re, im) prepared words
    double2* fs = reinterpret_cast<double2*>(ws + 2 * M);  // [M]
    double2* tab = fs + M;
    const double2* tws = tab + Tb::twist_off();
    const bool pre = a.in_spec != nullptr;
    const uint32_t i = blockIdx.x, lut = blockIdx.y, tid = threadIdx.x;
    const uint64_t Q = a.g.q;
    auto bar = []() { __syncthreads(); };

    for (uint32_t k = tid; k < Tb::size(); k += T) tab[k] = f.tab[k];
    const uint32_t set = a.lut_sel ? __ldg(a.lut_sel + lut) : lut;
    const uint64_t* in0 = a.in + set * a.in_lut_stride + static_cast<size_t>(2 * i) * 2 * N;
    const uint64_t* in1 = in0 + 2 * N;
    const double2* spec = nullptr;
    if (pre) {
        spec = a.in_spec + (static_cast<size_t>(set) * (a.in_count / 2) + i) * 2 * a.digits * M + tid;
    } else {
#pragma unroll
        for (uint32_t p = 0; p < 2; ++p) cmux_diff_words<N, T>(ws + p * M, in0, in1, p, a.g, tid);
    }
    __syncthreads();

    const uint32_t bit = __ldg(a.ctrl_bits + static_cast<size_t>(lut) * 8 + a.level);
    const double2* G = a.rgswf + static_cast<size_t>(bit) * a.rgsw_stride + tid;
    double2 y0[8], y1[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) y0[j] = y1[j] = make_double2(0.0, 0.0);
    for (uint32_t r = 0; r < 2 * a.digits; ++r) {
        double2 x[8];
        if (pre) {
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = __ldg(spec + static_cast<size_t>(r) * M + j * T);
        } else {
            cmux_digit_fft<LOGM>(fs, tid, tab, ws + (r & 1) * M, a.g.gbits, r >> 1, x, bar);
        }
        const double2* k0 = G + static_cast<size_t>(r) * 2 * M;
        const double2* k1 = k0 + M;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            cfma(y0[j], x[j], __ldg(k0 + j * T));
            cfma(y1[j], x[j], __ldg(k1 + j * T));
        }
        if (!pre) __syncthreads();
    }
    uint64_t* out = a.out + (static_cast<size_t>(lut) * (a.in_count / 2) + i) * 2 * N;
    fft_inverse_from_regs<LOGM>(
        fs, tid, tab, y0,
        [&](int j, uint32_t e, double2 v) {
            const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
            out[e] = add_mod(__ldg(in0 + e), double_to_mod(u.x * f.inv_m, f, Q), Q);
            out[e + M] = add_mod(__ldg(in0 + e + M), double_to_mod(u.y * f.inv_m, f, Q), Q);
        },
        bar);
    __syncthreads();
    fft_inverse_from_regs<LOGM>(
        fs, tid, tab, y1,
        [&](int j, uint32_t e, double2 v) {
            const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
            out[N + e] = add_mod(__ldg(in0 + N + e), double_to_mod(u.x * f.inv_m, f, Q), Q);
            out[N + e + M] = add_mod(__ldg(in0 + N + e + M), double_to_mod(u.y * f.inv_m, f, Q), Q);
        },
        bar);
}

// Spectra -> coefficient-domain polynomials mod Q, in place: CTA k inverse-transforms the
// spectrum of polynomial k (M double2 = N words) and overwrites it with its N coefficients.
// Every thread loads its spectrum slots before the transform's first barrier and stores only
// after its last one, so the in-place overwrite never races a load.
template <int LOGN>
__global__ void __launch_bounds__(LutFftCfg<LOGN>::T) k_spectra_to_coef(double2* buf, uint64_t Q, const FftKeyArgs f) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, T = M / 8;
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    double2* fs = reinterpret_cast<double2*>(smem);
    double2* tab = fs + M;
    const double2* tws = tab + Tb::twist_off();
    const uint32_t tid = threadIdx.x;
    for (uint32_t k = tid; k < Tb::size(); k += T) tab[k] = f.tab[k];
    double2* spec = buf + static_cast<size_t>(blockIdx.x) * M;
    double2 x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = spec[j * T + tid];
    __syncthreads();
    uint64_t* out = reinterpret_cast<uint64_t*>(spec);
    fft_inverse_from_regs<LOGM>(
        fs, tid, tab, x,
        [&](int j, uint32_t e, double2 v) {
            const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
            out[e] = double_to_mod(u.x * f.inv_m, f, Q);
            out[e + M] = double_to_mod(u.y * f.inv_m, f, Q);
        },
        []() { __syncthreads(); });
    (void)N;
}

// Coefficient-domain polynomials mod Q -> spectra (the row-spectrum form the FFT CMux reads):
// CTA k forward-transforms the centred polynomial coef[k] and stores its spectrum slot-major at
// out[k].  Out of place (the transform reads every coefficient of its polynomial).
template <int LOGN>
__global__ void __launch_bounds__(LutFftCfg<LOGN>::T) k_coef_to_spectra(const uint64_t* coef, double2* out,
                                                                          uint64_t Q, const FftKeyArgs f) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, T = M / 8;
    using Tb = FftTab<LOGM>;
    extern __shared__ __align__(16) uint64_t smem[];
    double2* fs = reinterpret_cast<double2*>(smem);
    double2* tab = fs + M;
    const uint32_t tid = threadIdx.x;
    for (uint32_t k = tid; k < Tb::size(); k += T) tab[k] = f.tab[k];
    __syncthreads();
    double2 x[8];
    fft_of_poly<LOGM>(fs, tid, tab, coef + static_cast<size_t>(blockIdx.x) * N, Q, x, []() { __syncthreads(); });
    store_spectrum<T>(out + static_cast<size_t>(blockIdx.x) * M, tid, x);
}

template <class K>
static cudaError_t opt_in_smem(K kernel, size_t bytes, size_t (&configured)[64]) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] >= bytes) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e == cudaSuccess) configured[dev] = bytes;
    return e;
}

template <int LOGN>
static cudaError_t trace_fft_launch(const TraceFftArgs& a, const FftKeyArgs& f, uint32_t count, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    const size_t smem = 2ull * N * sizeof(uint64_t) + (M + FftTab<LOGN - 1>::size()) * sizeof(double2);
    static size_t configured[64] = {};
    cudaError_t e = opt_in_smem(k_trace_ss_fft<LOGN>, smem, configured);
    if (e != cudaSuccess) return e;
    k_trace_ss_fft<LOGN><<<count, LutFftCfg<LOGN>::T, smem, s>>>(a, f);
    return cudaGetLastError();
}

template <int LOGN>
static cudaError_t cmux_fft_launch(const CmuxFftArgs& a, const FftKeyArgs& f, uint32_t luts, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    const size_t smem = 2ull * M * sizeof(uint2) + (M + FftTab<LOGN - 1>::size()) * sizeof(double2);
    static size_t configured[64] = {};
    cudaError_t e = opt_in_smem(k_cmux_level_fft<LOGN>, smem, configured);
    if (e != cudaSuccess) return e;
    const dim3 grid(a.in_count / 2, luts);
    k_cmux_level_fft<LOGN><<<grid, LutFftCfg<LOGN>::T, smem, s>>>(a, f);
    return cudaGetLastError();
}

template <int LOGN>
static cudaError_t pair_spectra_launch(const CmuxFftArgs& a, const FftKeyArgs& f, uint32_t sets, double2* out,
                                       cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2;
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    const size_t smem = 2ull * M * sizeof(uint2) + (M + FftTab<LOGN - 1>::size()) * sizeof(double2);
    static size_t configured[64] = {};
    cudaError_t e = opt_in_smem(k_cmux_pair_spectra<LOGN>, smem, configured);
    if (e != cudaSuccess) return e;
    const dim3 grid(a.in_count / 2, sets, 2 * a.digits);
    k_cmux_pair_spectra<LOGN><<<grid, LutFftCfg<LOGN>::T, smem, s>>>(a, f, out);
    return cudaGetLastError();
}

cudaError_t launch_cmux_pair_spectra(const CmuxFftArgs& a, const FftKeyArgs& f, uint32_t N, uint32_t sets,
                                     double2* out, cudaStream_t s) {
    if (sets == 0 || a.in_count < 2) return cudaSuccess;
    if (sets > 65535 || 2 * a.digits > 64 || a.in_count / 2 > 0x7fffffffu) return cudaErrorInvalidValue;
    switch (N) {
        case 1024: return pair_spectra_launch<10>(a, f, sets, out, s);
        case 2048: return pair_spectra_launch<11>(a, f, sets, out, s);
        case 4096: return pair_spectra_launch<12>(a, f, sets, out, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int LOGN>
static cudaError_t spectra_launch(double2* buf, uint64_t Q, const FftKeyArgs& f, size_t polys, cudaStream_t s) {
    constexpr uint32_t M = 1u << (LOGN - 1);
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    const size_t smem = (M + FftTab<LOGN - 1>::size()) * sizeof(double2);
    static size_t configured[64] = {};
    cudaError_t e = opt_in_smem(k_spectra_to_coef<LOGN>, smem, configured);
    if (e != cudaSuccess) return e;
    k_spectra_to_coef<LOGN><<<static_cast<unsigned>(polys), LutFftCfg<LOGN>::T, smem, s>>>(buf, Q, f);
    return cudaGetLastError();
}

cudaError_t launch_spectra_to_coef(double2* buf, uint64_t Q, const FftKeyArgs& f, uint32_t N, size_t polys,
                                   cudaStream_t s) {
    if (polys == 0) return cudaSuccess;
    if (polys > 0x7fffffffull) return cudaErrorInvalidValue;
    switch (N) {
        case 1024: return spectra_launch<10>(buf, Q, f, polys, s);
        case 2048: return spectra_launch<11>(buf, Q, f, polys, s);
        case 4096: return spectra_launch<12>(buf, Q, f, polys, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int LOGN>
static cudaError_t coef_spectra_launch(const uint64_t* coef, double2* out, uint64_t Q, const FftKeyArgs& f,
                                       size_t polys, cudaStream_t s) {
    constexpr uint32_t M = 1u << (LOGN - 1);
    if (f.tab_len != FftTab<LOGN - 1>::size()) return cudaErrorInvalidValue;
    const size_t smem = (M + FftTab<LOGN - 1>::size()) * sizeof(double2);
    static size_t configured[64] = {};
    cudaError_t e = opt_in_smem(k_coef_to_spectra<LOGN>, smem, configured);
    if (e != cudaSuccess) return e;
    k_coef_to_spectra<LOGN><<<static_cast<unsigned>(polys), LutFftCfg<LOGN>::T, smem, s>>>(coef, out, Q, f);
    return cudaGetLastError();
}

cudaError_t launch_coef_to_spectra(const uint64_t* coef, double2* out, uint64_t Q, const FftKeyArgs& f, uint32_t N,
                                   size_t polys, cudaStream_t s) {
    if (polys == 0) return cudaSuccess;
    if (polys > 0x7fffffffull) return cudaErrorInvalidValue;
    switch (N) {
        case 1024: return coef_spectra_launch<10>(coef, out, Q, f, polys, s);
        case 2048: return coef_spectra_launch<11>(coef, out, Q, f, polys, s);
        case 4096: return coef_spectra_launch<12>(coef, out, Q, f, polys, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_trace_ss_fft(const TraceFftArgs& a, const FftKeyArgs& f, uint32_t N, uint32_t count,
                                cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    if (a.rounds > 16 || a.digits_ht == 0 || a.digits_ss == 0) return cudaErrorInvalidValue;
    switch (N) {
        case 1024: return trace_fft_launch<10>(a, f, count, s);
        case 2048: return trace_fft_launch<11>(a, f, count, s);
        case 4096: return trace_fft_launch<12>(a, f, count, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_cmux_level_fft(const CmuxFftArgs& a, const FftKeyArgs& f, uint32_t N, uint32_t luts,
                                  cudaStream_t s) {
    if (luts == 0) return cudaSuccess;
    if (a.in_count < 2 || a.digits == 0 || a.digits * static_cast<uint32_t>(a.g.gbits) > 32)
        return cudaErrorInvalidValue;
    if (luts > 65535 || (a.in_spec && a.level != 0)) return cudaErrorInvalidValue;
    switch (N) {
        case 1024: return cmux_fft_launch<10>(a, f, luts, s);
        case 2048: return cmux_fft_launch<11>(a, f, luts, s);
        case 4096: return cmux_fft_launch<12>(a, f, luts, s);
        default: return cudaErrorInvalidValue;
    }
}

DigitPrep make_digit_prep(uint64_t q, const Gadget& g, uint32_t digits) {
    DigitPrep d{};
    d.q = q;
    d.qhalf = q >> 1;
    d.ign = g.ign;
    d.gbits = g.gbits;
    uint64_t offset = 0;
    for (uint32_t k = 0; k < digits; ++k) offset += uint64_t(1) << (g.gbits * k + g.gbits - 1);
    d.round_c = (g.ign ? (uint64_t(1) << (g.ign - 1)) : 0) + (offset << g.ign);
    return d;
}

}  // namespace cbs
