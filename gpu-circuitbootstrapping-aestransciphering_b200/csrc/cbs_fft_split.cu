// cbs_fft_split.cu -- exact blind rotation with FP64 FFT products of key limbs.
//
// The reference's split-FFT CBS backend (bitwise/src/cirbts/cirbts-init.cu:1084-1140 sizes the
// limbs as 50 - (log2 Bg + log2 N + log2 digitsG2) bits, cirbts-init.cu:1255-1280 cuts the key
// into limbs and transforms them, cirbts-bootstrap.cu:939-1085 runs, per LWE coefficient and per
// limb, the digit x limb product, one inverse transform and an add scaled by 2^(limb_bits l)
// mod Q).  Every product of a gadget digit polynomial and a key limb polynomial, summed over the
// 2 digits key rows and multiplied by X^a - 1, has integer coefficients far below 2^53, so the
// FP64 transform rounds each one back to its exact value; the limb results are reduced mod Q and
// combined.  The accumulator is therefore the exact GINX accumulator of k_blind_rotate
// (cirbts-batch.cu:3293-4629), and the MV outputs are bit-identical to the exact NTT kernel's.
//
// Differences from the reference's form, kept because they are faster here: limbs are balanced
// (signed, one bit of headroom more than unsigned limbs, so limb widths are equalised as
// ceil(log2 Q / limbs)); all n steps run in one kernel with the accumulator resident in shared
// memory (k_blind_rotate_fft's layout and offset-form accumulator); the digit spectra are
// computed once per step and held in registers across the limbs; X^a - 1 is applied to each
// limb's output spectrum before its inverse transform.
#include <algorithm>
#include <cmath>
#include <complex>
#include <thread>
#include <vector>

#include "cbs_kernels.cuh"
#include "common.cuh"
#include "fft_core.cuh"
#include "fft_kernels.cuh"
#include "fft_ops.cuh"

namespace cbs {

template <int LOGN>
struct BrSplitCfg {
    static constexpr uint32_t T = (1u << LOGN) / 8;
    static constexpr int MIN_BLOCKS = LOGN <= 10 ? 2 : 1;
};

// Two halves of M/8 threads per CTA (k_blind_rotate_fft's organisation).  Per step (MB = 1) or
// group of two coefficients (MB = 2):
//  1. digits of each half's accumulator polynomial, packed biased pairs in shared memory;
//  2. half h forward-transforms its DIG digit polynomials into registers;
//  3. per limb l: both key columns of rows 2d + h, limb l (MB = 2: the combined keys
//     c0 (K0 + c1 K01) + c1 K1, one column at a time), against the digit spectra; the halves
//     swap partial sums so half h holds output h; MB = 1: times psi^a - 1; inverse transform;
//     each coefficient rounds to the exact integer limb product, is scaled by 2^(lb l) mod Q and
//     added to the accumulator position this thread owns.
template <int LOGN, bool WIDE, int DIG, int MB>
__global__ void __launch_bounds__(BrSplitCfg<LOGN>::T, BrSplitCfg<LOGN>::MIN_BLOCKS)
    k_blind_rotate_fft_split(const BlindRotateArgs a, const FftKeyArgs f, const SplitKeyArgs sk) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, T = 2 * TH, TWO_N = 2 * N;
    using Tb = FftTab<LOGM>;
    using DigT = typename DigitPair<WIDE>::T;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* acc = smem;                                           // [2][N]
    double2* fs = reinterpret_cast<double2*>(smem + 2 * N);         // [2][M]
    double2* tab = fs + 2 * M;                                      // FftTab<LOGM>
    DigT* dig = reinterpret_cast<DigT*>(tab + Tb::size());          // [2][DIG][M] digit pairs
    double2* cbuf = reinterpret_cast<double2*>(dig + 2 * DIG * M);  // MB = 2: [2][8][T] c_i per slot
    const double2* tws = tab + Tb::twist_off();
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const uint32_t h = tid / TH, ht = tid % TH;
    int64_t* my_acc = reinterpret_cast<int64_t*>(acc) + h * N;
    double2* my_fs = fs + h * M;
    const uint64_t Q = a.t.q;
    const int gbits = a.g.gbits;
    int64_t offset = 0;
    for (int k = 0; k < DIG; ++k) offset += static_cast<int64_t>(1) << (gbits * k + gbits - 1);
    const int ign = a.g.ign;
    const uint64_t qhalf = Q >> 1;
    // offset form of the accumulator (k_blind_rotate_fft): y = centre(x) + round_c in [lo_b, hi_b),
    // so the prepared digit word is y >> ign
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
    // one rounded limb-product coefficient (exact, |v| < 2^bound_bits < Q/2) scaled by 2^(lb l)
    // mod Q: the centred value itself for limb 0, a residue in [0, Q) for the others
    // (offset_add corrects either by one +-Q)
    auto limb_term = [&](double u, uint32_t l, uint64_t pw, uint64_t pws) -> int64_t {
        const int64_t v = __double2ll_rn(u * f.inv_m);
        if (l == 0) return v;
        const uint64_t vm = static_cast<uint64_t>(v < 0 ? v + Qs : v);
        return static_cast<int64_t>(mul_shoup(vm, pw, pws, Q));
    };
    const uint32_t limbs = sk.limbs;
    const int32_t dbias = 1 << (gbits - 1);
    const uint32_t fmask = (1u << gbits) - 1u;
    const uint64_t* arow = a.a + static_cast<size_t>(ct) * a.a_stride;
    // key polynomials per step and limb: [subsets][2*DIG rows][2 columns]
    constexpr uint32_t PER_STEP = (MB == 1 ? 1 : 3) * 4 * DIG;
    const uint32_t steps = (a.n + MB - 1) / MB;
    for (uint32_t step = 0; step < steps; ++step) {
        // mask exponents of the step's coefficients (0 past n: X^0 - 1 = 0 drops the term)
        uint32_t at[MB];
#pragma unroll
        for (int i = 0; i < MB; ++i) {
            const uint32_t idx = step * MB + i;
            at[i] = idx < a.n ? special_ms_f(__ldg(arow + idx), TWO_N, a.q_lwe, a.bitwidth) : 0u;
        }
        if constexpr (MB == 2) {
            // c_i(psi_s) = psi_s^(a_i) - 1 for the thread's 8 slots, thread-private in shared
            // memory for the step (the combined key c0 (K0 + c1 K01) + c1 K1 needs them per limb)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const uint32_t mb_i = mult_base<LOGN>(ht, at[i]);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const double2 w = zeta_pow<LOGN>(tws, slot_exp<LOGN>(mb_i, at[i], j));
                    cbuf[(i * 8 + j) * T + tid] = make_double2(w.x - 1.0, w.y);
                }
            }
        }
        // 1. digits of this half's polynomial (positions ht + j*TH, owned by this thread)
        for (uint32_t e = ht; e < M; e += TH) {
            const uint64_t wr = static_cast<uint64_t>(my_acc[e]) >> ign;
            const uint64_t wi = static_cast<uint64_t>(my_acc[e + M]) >> ign;
            DigT* dst = dig + h * DIG * M + e;
#pragma unroll
            for (int d = 0; d < DIG; ++d)
                dst[d * M] = DigitPair<WIDE>::pack(static_cast<uint32_t>(wr >> (gbits * d)) & fmask,
                                                   static_cast<uint32_t>(wi >> (gbits * d)) & fmask);
        }
        half_bar();
        // 2. digit spectra, held for every limb
        double2 x[DIG][8];
#pragma unroll
        for (int d = 0; d < DIG; ++d) {
            const DigT* dsrc = dig + (h * DIG + d) * M;
            fft_forward_to_regs<LOGM>(
                my_fs, ht, tab,
                [&](int j, uint32_t e) {
                    return cmul(DigitPair<WIDE>::unpack(dsrc[e], dbias), twist_at<LOGM>(tws, j, e));
                },
                x[d], half_bar);
            half_bar();
        }
        const uint32_t mbase = mult_base<LOGN>(ht, at[0]);
        const double2* ek = sk.bskx + static_cast<size_t>(step) * limbs * PER_STEP * M + ht;
        // 3. one product, swap and inverse transform per limb
#pragma unroll 1
        for (uint32_t l = 0; l < limbs; ++l) {
            const double2* el = ek + static_cast<size_t>(l) * PER_STEP * M;
            // 2^(lb l) mod Q by selects on the uniform l (an indexed kernel-parameter array
            // would be copied to local memory)
            const uint64_t pw = l == 1 ? sk.pw[1] : (l == 2 ? sk.pw[2] : sk.pw[3]);
            const uint64_t pws = l == 1 ? sk.pws[1] : (l == 2 ? sk.pws[2] : sk.pws[3]);
            // mb = 2, column c of this half's partial product: sum over d of the digit spectrum
            // times the combined key c0 (K0 + c1 K01) + c1 K1 of row 2d + h, column c (subsets
            // {0} {1} {0,1} at spectrum offsets 0, 4 DIG M, 8 DIG M)
            auto column = [&](uint32_t c, double2 (&y)[8]) {
                constexpr size_t KS = static_cast<size_t>(4) * DIG * M;
#pragma unroll
                for (int j = 0; j < 8; ++j) y[j] = make_double2(0.0, 0.0);
#pragma unroll
                for (int d = 0; d < DIG; ++d) {
                    const double2* kc = el + (static_cast<size_t>(2 * d + h) * 2 + c) * M;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const double2 c0 = cbuf[j * T + tid], c1 = cbuf[(8 + j) * T + tid];
                        double2 t = __ldg(kc + j * TH);
                        cfma(t, c1, __ldg(kc + 2 * KS + j * TH));
                        double2 r = cmul(c0, t);
                        cfma(r, c1, __ldg(kc + KS + j * TH));
                        cfma(y[j], x[d][j], r);
                    }
                }
            };
            double2 y0[8];
            if constexpr (MB == 1) {
                // both columns together: twice the key loads in flight (faster one-bit, where the
                // registers allow it)
                double2 y1[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) y0[j] = y1[j] = make_double2(0.0, 0.0);
#pragma unroll
                for (int d = 0; d < DIG; ++d) {
                    const double2* k0 = el + static_cast<size_t>(2 * d + h) * 2 * M;  // row 2d + h
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        cfma(y0[j], x[d][j], __ldg(k0 + j * TH));
                        cfma(y1[j], x[d][j], __ldg(k0 + M + j * TH));
                    }
                }
                // the previous limb's inverse transform (or the forward passes) no longer reads fs
                __syncthreads();
#pragma unroll
                for (int j = 0; j < 8; ++j) my_fs[cswz(8 * ht + j)] = h ? y0[j] : y1[j];
                __syncthreads();
                const double2* take = fs + (1 - h) * M;
#pragma unroll
                for (int j = 0; j < 8; ++j) y0[j] = cadd(h ? y1[j] : y0[j], take[cswz(8 * ht + j)]);
            } else {
                // the other half's output column first (its key loads overlap the barrier), then
                // this half's own column while the other half's partial sums land: one column of
                // accumulators is live at a time (the combined keys need the registers)
                column(1 - h, y0);
                __syncthreads();  // the previous limb's inverse transform no longer reads fs
#pragma unroll
                for (int j = 0; j < 8; ++j) my_fs[cswz(8 * ht + j)] = y0[j];
                column(h, y0);
                __syncthreads();
                const double2* take = fs + (1 - h) * M;
#pragma unroll
                for (int j = 0; j < 8; ++j) y0[j] = cadd(y0[j], take[cswz(8 * ht + j)]);
            }
            __syncthreads();
            if constexpr (MB == 1) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const double2 w = zeta_pow<LOGN>(tws, slot_exp<LOGN>(mbase, at[0], j));
                    y0[j] = cmul(y0[j], make_double2(w.x - 1.0, w.y));
                }
            }
            fft_inverse_from_regs<LOGM>(
                my_fs, ht, tab, y0,
                [&](int j, uint32_t e, double2 v) {
                    const double2 u = cmulc(v, twist_at<LOGM>(tws, j, e));
                    my_acc[e] = offset_add(my_acc[e], limb_term(u.x, l, pw, pws), lo_b, hi_b, Qs);
                    my_acc[e + M] = offset_add(my_acc[e + M], limb_term(u.y, l, pw, pws), lo_b, hi_b, Qs);
                },
                half_bar);
        }
    }
    __syncthreads();

    // finalize (cirbts-batch.cu:2622-2642) and the MV split ct_j = acc * X^-j, as
    // k_blind_rotate_fft; the caller transforms mv_out to the NTT domain
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

cudaError_t ntt_forward(uint64_t* out, const uint64_t* in, const uint64_t* tw, const uint64_t* tws,
                        const cbs_dmodulus* mod, size_t dim, size_t batch, cudaStream_t s);

template <int LOGN, bool WIDE, int DIG, int MB>
static cudaError_t br_split_launch(const BlindRotateArgs& a, const FftKeyArgs& f, const SplitKeyArgs& k,
                                   uint32_t batch, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN, M = N / 2, T = BrSplitCfg<LOGN>::T;
    const size_t smem = 2ull * N * sizeof(uint64_t) + (2ull * M + FftTab<LOGN - 1>::size()) * sizeof(double2) +
                        2ull * DIG * M * sizeof(typename DigitPair<WIDE>::T) +
                        (MB == 2 ? 2ull * 8 * T * sizeof(double2) : 0);
    static size_t configured[64] = {};  // per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_blind_rotate_fft_split<LOGN, WIDE, DIG, MB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_blind_rotate_fft_split<LOGN, WIDE, DIG, MB><<<batch, T, smem, s>>>(a, f, k);
    return cudaGetLastError();
}

template <int LOGN, bool WIDE>
static cudaError_t br_split_launch(const BlindRotateArgs& a, const FftKeyArgs& f, const SplitKeyArgs& k,
                                   uint32_t batch, uint32_t mb, cudaStream_t s) {
    if (mb == 2) {
        switch (a.digits) {
            case 2: return br_split_launch<LOGN, WIDE, 2, 2>(a, f, k, batch, s);
            case 3: return br_split_launch<LOGN, WIDE, 3, 2>(a, f, k, batch, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (a.digits) {
        case 2: return br_split_launch<LOGN, WIDE, 2, 1>(a, f, k, batch, s);
        case 3: return br_split_launch<LOGN, WIDE, 3, 1>(a, f, k, batch, s);
        case 4: return br_split_launch<LOGN, WIDE, 4, 1>(a, f, k, batch, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_blind_rotate_fft_split(const BlindRotateArgs& a, const FftKeyArgs& f, const SplitKeyArgs& k,
                                          const cbs_dmodulus* d_mod, uint32_t N, uint32_t batch, uint32_t mb,
                                          cudaStream_t s) {
    if (batch == 0) return cudaSuccess;
    if (a.g.gbits < 1 || a.g.gbits > 24 || a.digits < 2 || a.digits > (mb == 2 ? 3u : 4u)) return cudaErrorInvalidValue;
    if (mb != 1 && mb != 2) return cudaErrorInvalidValue;
    if (k.limbs < 1 || k.limbs > kMaxSplitLimbs || k.bskx == nullptr) return cudaErrorInvalidValue;
    if (f.tab_len != (N == 1024 ? FftTab<9>::size() : FftTab<10>::size())) return cudaErrorInvalidValue;
    const bool wide = wide_digits(a.g.gbits);
    cudaError_t e;
    switch (N) {
        case 1024:
            e = wide ? br_split_launch<10, true>(a, f, k, batch, mb, s) : br_split_launch<10, false>(a, f, k, batch, mb, s);
            break;
        case 2048:
            e = wide ? br_split_launch<11, true>(a, f, k, batch, mb, s) : br_split_launch<11, false>(a, f, k, batch, mb, s);
            break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    return ntt_forward(a.mv_out, a.mv_out, a.t.rp, a.t.rps, d_mod, N, static_cast<size_t>(batch) * a.num_lut * 2, s);
}

// ---- host side ----

static uint32_t bit_length(uint64_t v) {
    uint32_t b = 0;
    while (b < 64 && (v >> b) != 0) ++b;
    return b;
}

bool split_plan(uint32_t N, uint64_t Q, int gbits, uint32_t digits, uint32_t mb, SplitPlan& out) {
    if (N < 2 || (N & (N - 1)) || Q < 3 || gbits < 1 || digits < 1 || mb < 1 || mb > 2) return false;
    const uint32_t logn = bit_length(N) - 1, logq = bit_length(Q);
    const uint32_t log_rows = bit_length(2 * digits - 1);  // ceil(log2(2 digits))
    // |limb| <= 2^(lb-1), |digit| <= 2^(g-1), N * 2 digits terms, times the monomial factor: X^a - 1
    // (L1 norm 2, one bit) for mb = 1, c0 + c1 + c0 c1 (L1 norm 2 + 2 + 4, three bits) for mb = 2:
    // bound_bits = lb + g - 2 + log2 N + ceil(log2(2 digits)) + mono_bits, kept <= 50 (the
    // reference's margin)
    const uint32_t mono_bits = mb == 1 ? 1 : 3;
    const int lb_max = 52 - gbits - static_cast<int>(logn) - static_cast<int>(log_rows) - static_cast<int>(mono_bits);
    if (lb_max < 2) return false;
    const uint32_t limbs = (logq + static_cast<uint32_t>(lb_max) - 1) / static_cast<uint32_t>(lb_max);
    if (limbs < 1 || limbs > kMaxSplitLimbs) return false;
    const uint32_t lb = (logq + limbs - 1) / limbs;
    const uint32_t bound = lb + static_cast<uint32_t>(gbits) - 2 + logn + log_rows + mono_bits;
    // the rounded limb product must also sit below Q/2 (it is added as a centred residue):
    // 2^bound <= 2^(logq - 2) <= Q/2
    if (bound > 50 || bound + 2 > logq) return false;
    out.limbs = limbs;
    out.limb_bits = lb;
    out.bound_bits = bound;
    return true;
}

void keys_to_fft_limbs_host(const host::NttTables& t, const uint64_t* keys_ntt, size_t count, uint32_t per_step,
                            const SplitPlan& plan, std::vector<double2>& out) {
    const uint32_t N = t.n, M = N / 2, L = plan.limbs, lb = plan.limb_bits;
    const uint64_t Q = t.q;
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<cld> w(M / 2), twist(M);
    for (uint32_t e = 0; e < M / 2; ++e) w[e] = std::polar(1.0L, 2.0L * pi * e / M);
    for (uint32_t e = 0; e < M; ++e) twist[e] = std::polar(1.0L, pi * e / N);
    out.assign(count * L * M, make_double2(0, 0));
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th) {
        pool.emplace_back([&, th] {
            std::vector<uint64_t> c(N);
            std::vector<int64_t> v(N), limb(N);
            std::vector<cld> z(M);
            for (size_t k = th; k < count; k += nth) {
                std::copy(keys_ntt + k * N, keys_ntt + (k + 1) * N, c.begin());
                host::ntt_inverse_host(c.data(), t);
                for (uint32_t e = 0; e < N; ++e)
                    v[e] = c[e] > Q / 2 ? -static_cast<int64_t>(Q - c[e]) : static_cast<int64_t>(c[e]);
                const size_t step = k / per_step, within = k % per_step;
                for (uint32_t l = 0; l < L; ++l) {
                    // balanced limb l; the last limb takes the remaining high part
                    for (uint32_t e = 0; e < N; ++e) {
                        if (l + 1 < L) {
                            const int64_t half = int64_t(1) << (lb - 1);
                            const int64_t r = ((v[e] + half) & ((int64_t(1) << lb) - 1)) - half;
                            limb[e] = r;
                            v[e] = (v[e] - r) >> lb;
                        } else {
                            limb[e] = v[e];
                        }
                    }
                    for (uint32_t e = 0; e < M; ++e)
                        z[e] = cld(static_cast<long double>(limb[e]), static_cast<long double>(limb[e + M])) *
                               twist[e];
                    // slot s stored at (s % 8) * (M / 8) + s / 8 (the register order of the
                    // thread that consumes it, as keys_to_fft_host)
                    host_dif(z, w);
                    const size_t o = (step * L + l) * per_step + within;
                    for (uint32_t e = 0; e < M; ++e)
                        out[o * M + (e % 8) * (M / 8) + e / 8] =
                            make_double2(static_cast<double>(z[e].real()), static_cast<double>(z[e].imag()));
                }
            }
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace cbs
