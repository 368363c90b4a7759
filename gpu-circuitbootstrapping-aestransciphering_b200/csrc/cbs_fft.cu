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
#include <vector>

#include "cbs_kernels.cuh"
#include "common.cuh"
#include "fft_core.cuh"
#include "fft_kernels.cuh"

namespace cbs {

__device__ __forceinline__ int32_t digit_signed(uint64_t x, const Gadget& g, uint32_t d) {
    int64_t v = gadget_prepare(x, g);
    int32_t r = 0;
    for (uint32_t i = 0; i <= d; ++i) r = peel_digit(v, g.gbits);
    return r;
}

// round(v) mod Q for |v| < 2^62 * 2^30 (v is the FP64 result of an integer-valued product)
__device__ __forceinline__ uint64_t double_to_mod(double v, uint64_t Q, const uint64_t* __restrict__ pow2,
                                                  const uint64_t* __restrict__ pow2s) {
    const long long bits = __double_as_longlong(v);
    const int ex = static_cast<int>((bits >> 52) & 0x7ff);
    const bool neg = bits < 0;
    uint64_t r;
    if (ex < 1075) {  // |v| < 2^52: round to the nearest integer directly
        const long long i = __double2ll_rn(v);
        const uint64_t a = static_cast<uint64_t>(i < 0 ? -i : i);
        r = a;  // a < 2^52 < Q
        return (i < 0 && r) ? Q - r : r;
    }
    const int e = ex - 1075;  // v = +-mantissa * 2^e exactly
    const uint64_t mant = (static_cast<uint64_t>(bits) & ((1ull << 52) - 1)) | (1ull << 52);  // < 2^53 < Q
    r = mul_shoup(mant, __ldg(pow2 + e), __ldg(pow2s + e), Q);
    return (neg && r) ? Q - r : r;
}

template <uint32_t N, uint32_t T>
__device__ __forceinline__ void rotate_add_f(uint64_t* acc, const uint64_t* t, uint32_t e, uint32_t tid, uint64_t q) {
#pragma unroll 4
    for (uint32_t k = 0; k < N / T; ++k) {
        const uint32_t i = tid + k * T;
        const uint32_t s = (i + 2 * N - e) & (2 * N - 1);
        uint64_t v = (s < N) ? t[s] : t[s - N];
        if (s >= N) v = v ? q - v : 0;
        acc[i] = add_mod(acc[i], sub_mod(v, t[i], q), q);
    }
}

// Two 128-thread halves per CTA (N = 2048): half h owns accumulator polynomial h.  Per step
// each half forward-transforms the digits of its polynomial and multiplies them against
// both key columns; the halves then swap partial sums through shared memory so that half 0
// holds the full spectrum of output 0 and half 1 that of output 1, inverse-transform them
// side by side, and all threads rotate-add both outputs.
template <int LOGN>
__global__ void __launch_bounds__((1 << LOGN) / 8, 2) k_blind_rotate_fft(const BlindRotateArgs a,
                                                                        const FftKeyArgs f) {
    constexpr int LOGM = LOGN - 1;
    constexpr uint32_t N = 1u << LOGN, M = N / 2, TH = M / 8, T = 2 * TH, TWO_N = 2 * N;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* acc = smem;                                      // [2][N]
    uint64_t* tb = smem + 2 * N;                               // [2][N]
    double2* fs = reinterpret_cast<double2*>(smem + 4 * N);    // [2][M]
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const uint32_t h = tid / TH, ht = tid % TH;
    uint64_t* my_acc = acc + h * N;
    double2* my_fs = fs + h * M;
    const uint64_t Q = a.t.q;

    {
        const uint32_t bt = special_ms_f(a.b[ct], TWO_N, a.q_lwe, a.bitwidth);
        for (uint32_t i = tid; i < N; i += T) {
            acc[i] = 0;
            const uint32_t s = (i + bt) & (TWO_N - 1);
            const uint64_t v = (s < N) ? a.tv[s] : a.tv[s - N];
            acc[N + i] = (s < N) ? v : (v ? Q - v : 0);
        }
    }
    __syncthreads();

    const uint32_t l2 = 2 * a.digits;
    const uint64_t* arow = a.a + static_cast<size_t>(ct) * a.a_stride;
    for (uint32_t step = 0; step < a.n; ++step) {
        const uint32_t at = special_ms_f(__ldg(arow + step), TWO_N, a.q_lwe, a.bitwidth);
        const double2* ek = f.bskf + static_cast<size_t>(step) * l2 * 2 * M;
        double2 y0[8], y1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) y0[j] = y1[j] = make_double2(0.0, 0.0);
        for (uint32_t d = 0; d < a.digits; ++d) {
            const uint32_t r = 2 * d + h;  // key row: digit d of polynomial h
            double2 x[8];
            fft_forward_to_regs<LOGM>(
                my_fs, ht, f.tw,
                [&](uint32_t e) {
                    const double re = static_cast<double>(digit_signed(my_acc[e], a.g, d));
                    const double im = static_cast<double>(digit_signed(my_acc[e + M], a.g, d));
                    return cmul(make_double2(re, im), __ldg(f.twist + e));
                },
                x);
            const double2* k0 = ek + static_cast<size_t>(r) * 2 * M + 8 * ht;
            const double2* k1 = k0 + M;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                cfma(y0[j], x[j], __ldg(k0 + j));
                cfma(y1[j], x[j], __ldg(k1 + j));
            }
            __syncthreads();
        }
        // swap partial sums: half 0 keeps output 0, half 1 keeps output 1
        {
            double2* give = my_fs + 8 * ht;
#pragma unroll
            for (int j = 0; j < 8; ++j) give[j] = h ? y0[j] : y1[j];
            __syncthreads();
            const double2* take = fs + (1 - h) * M + 8 * ht;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const double2 t = take[j];
                if (h) y1[j] = cadd(y1[j], t);
                else y0[j] = cadd(y0[j], t);
            }
            __syncthreads();
        }
        uint64_t* my_tb = tb + h * N;
#pragma unroll
        for (int j = 0; j < 8; ++j) y0[j] = h ? y1[j] : y0[j];  // register-wise select, no indexing
        fft_inverse_from_regs<LOGM>(my_fs, ht, f.tw, y0, [&](uint32_t e, double2 v) {
            const double2 u = cmulc(v, __ldg(f.twist + e));
            my_tb[e] = double_to_mod(u.x * f.inv_m, Q, f.pow2, f.pow2s);
            my_tb[e + M] = double_to_mod(u.y * f.inv_m, Q, f.pow2, f.pow2s);
        });
        __syncthreads();
        rotate_add_f<N, T>(acc, tb, at, tid, Q);
        rotate_add_f<N, T>(acc + N, tb + N, at, tid, Q);
        __syncthreads();
    }

    // finalize (cirbts-batch.cu:2622-2642) and the MV split ct_j = acc * X^-j in the
    // coefficient domain; the caller transforms mv_out to the NTT domain
    for (uint32_t i = tid; i < N; i += T) {
        acc[i] = mul_shoup(acc[i], a.t.n_inv, a.t.n_inv_s, Q);
        uint64_t v = mul_shoup(acc[N + i], a.t.n_inv, a.t.n_inv_s, Q);
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

template <int LOGN>
static cudaError_t br_fft_launch(const BlindRotateArgs& a, const FftKeyArgs& f, uint32_t batch, cudaStream_t s) {
    constexpr uint32_t N = 1u << LOGN;
    const size_t smem = 6ull * N * sizeof(uint64_t);
    static size_t configured = 0;
    if (configured < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_blind_rotate_fft<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    k_blind_rotate_fft<LOGN><<<batch, N / 8, smem, s>>>(a, f);
    return cudaGetLastError();
}

cudaError_t launch_blind_rotate_fft(const BlindRotateArgs& a, const FftKeyArgs& f, const cbs_dmodulus* d_mod,
                                    uint32_t N, uint32_t batch, cudaStream_t s) {
    if (batch == 0) return cudaSuccess;
    cudaError_t e;
    switch (N) {
        case 1024: e = br_fft_launch<10>(a, f, batch, s); break;
        case 2048: e = br_fft_launch<11>(a, f, batch, s); break;
        case 4096: e = br_fft_launch<12>(a, f, batch, s); break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    return ntt_forward(a.mv_out, a.mv_out, a.t.rp, a.t.rps, d_mod, N, static_cast<size_t>(batch) * a.num_lut * 2, s);
}

// ---- host side: FFT-domain key material ----

using cld = std::complex<long double>;

static void host_dif(std::vector<cld>& a, const std::vector<cld>& w) {
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

void fft_tables_host(uint32_t N, std::vector<double2>& tw, std::vector<double2>& twist) {
    const uint32_t M = N / 2;
    const long double pi = 3.141592653589793238462643383279502884L;
    tw.resize(M / 2);
    for (uint32_t e = 0; e < M / 2; ++e) {
        const long double ang = 2.0L * pi * e / M;
        tw[e] = make_double2(static_cast<double>(cosl(ang)), static_cast<double>(sinl(ang)));
    }
    twist.resize(M);
    for (uint32_t e = 0; e < M; ++e) {
        const long double ang = pi * e / N;
        twist[e] = make_double2(static_cast<double>(cosl(ang)), static_cast<double>(sinl(ang)));
    }
}

// NTT-domain key polynomials [count][N] (normal form, mod Q) -> FFT spectra [count][M]
void keys_to_fft_host(const host::NttTables& t, const uint64_t* keys_ntt, size_t count, std::vector<double2>& out) {
    const uint32_t N = t.n, M = N / 2;
    const uint64_t Q = t.q;
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<cld> w(M / 2), twist(M);
    for (uint32_t e = 0; e < M / 2; ++e) w[e] = std::polar(1.0L, 2.0L * pi * e / M);
    for (uint32_t e = 0; e < M; ++e) twist[e] = std::polar(1.0L, pi * e / N);
    out.assign(count * M, make_double2(0, 0));
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th) {
        pool.emplace_back([&, th] {
            std::vector<uint64_t> c(N);
            std::vector<cld> z(M);
            for (size_t k = th; k < count; k += nth) {
                std::copy(keys_ntt + k * N, keys_ntt + (k + 1) * N, c.begin());
                host::ntt_inverse_host(c.data(), t);
                for (uint32_t e = 0; e < M; ++e) {
                    const long double re = c[e] > Q / 2 ? -static_cast<long double>(Q - c[e]) : static_cast<long double>(c[e]);
                    const long double im =
                        c[e + M] > Q / 2 ? -static_cast<long double>(Q - c[e + M]) : static_cast<long double>(c[e + M]);
                    z[e] = cld(re, im) * twist[e];
                }
                host_dif(z, w);
                for (uint32_t e = 0; e < M; ++e)
                    out[k * M + e] = make_double2(static_cast<double>(z[e].real()), static_cast<double>(z[e].imag()));
            }
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace cbs
