// fft_kernels.cuh -- FP64 FFT blind-rotation backend: launch interface and host key prep.
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <vector>

#include "cbs_kernels.cuh"
#include "host_math.h"

namespace cbs {

struct FftKeyArgs {
    const double2* bskf;    // [n][2*digits][2][N/2] key spectra (forward-FFT slot order)
    const double2* tab;     // FftTab<log2(N/2)> layout: twiddles of every pass + half twist table
    uint32_t tab_len;       // entries of tab
    const uint64_t* pow2;   // [64] 2^e mod Q
    const uint64_t* pow2s;  // Shoup quotients of pow2
    double inv_m;           // 1 / (N/2)
    double q_hi, q_lo;      // Q = q_hi + q_lo exactly (q_hi = Q rounded to a double, |q_lo| <= 1)
    double inv_q;           // 1 / Q rounded
};

// Balanced gadget digits by the offset trick: (centred x + round_c) >> ign holds every digit
// plus 2^(gbits-1) in its bit field k (see prepared_offset in cbs_fft.cu).
struct DigitPrep {
    uint64_t q, qhalf;
    uint64_t round_c;  // 2^(ign-1) + (sum_k 2^(gbits k + gbits - 1)) << ign
    int ign, gbits;
};

// HomTrace + SchemeSwitch on coefficient-domain MV RLWEs with FFT key switching.
struct TraceFftArgs {
    const uint64_t* mv;     // [count][2][N] coefficient domain (a, b)
    double2* rgswf;         // [count][2 row types][2 polys][N/2] spectra, slot-major
    uint32_t rounds;
    uint32_t kinv[16];      // inverse mod 2N of the automorphism exponent N/2^r + 1 of round r
    const double2* htf;     // [rounds][digits_ht][3][N/2] key spectra: k0_hi, k0_lo, k1
    const double2* ssf;     // [digits_ss][3][N/2]
    uint64_t split_pow, split_pow_s;  // 2^kTraceKeySplitBits mod Q and its Shoup quotient
    DigitPrep g_ht, g_ss;
    uint32_t digits_ht, digits_ss;
};

// One LUT-tree level of FFT CMuxes on coefficient-domain RLWEs.
struct CmuxFftArgs {
    const uint64_t* in;           // level input: [sets][in_count][2][N] coefficient domain
    uint64_t in_lut_stride;       // words between input sets
    const uint32_t* lut_sel;      // input set of each LUT (level 0: table id); null = the LUT index
    uint64_t* out;                // [luts][in_count/2][2][N] coefficient domain
    uint32_t in_count;
    const double2* rgswf;         // [bits][digits][2][2][N/2] spectra (TraceFftArgs::rgswf)
    uint64_t rgsw_stride;         // spectra entries per bit
    const uint32_t* ctrl_bits;    // [luts][8] bit index of the control for each level
    uint32_t level;
    DigitPrep g;
    uint32_t digits;
    // level 0 over fixed tables: [sets][in_count/2][2*digits][N/2] digit spectra of
    // in[2i+1] - in[2i] from launch_cmux_pair_spectra (null: computed in the CMux)
    const double2* in_spec;
};

// Exact blind rotation over FP64 products of key limbs: each key polynomial k (centred) is
// cut into `limbs` balanced limbs of `limb_bits` bits, k = sum_l 2^(limb_bits l) k_l, and the
// limb spectra of one step are stored [limbs][2*digits][2][N/2] (slot-major, as bskf).
constexpr uint32_t kMaxSplitLimbs = 4;
struct SplitPlan {
    uint32_t limbs = 0, limb_bits = 0;
    uint32_t bound_bits = 0;  // log2 of the bound on every rounded limb-product coefficient
};
struct SplitKeyArgs {
    const double2* bskx;                 // [n][limbs][2*digits][2][N/2] limb spectra
    uint32_t limbs;
    uint64_t pw[kMaxSplitLimbs];         // 2^(limb_bits l) mod Q
    uint64_t pws[kMaxSplitLimbs];        // their Shoup quotients
};
// the limb split for ring N, modulus Q, a gadget of `digits` digits of gbits bits and the
// grouping mb (1 or 2): false when no split of at most kMaxSplitLimbs limbs keeps the products
// below 2^50 and Q / 2
bool split_plan(uint32_t N, uint64_t Q, int gbits, uint32_t digits, uint32_t mb, SplitPlan& out);
// key polynomials [count][N] (NTT domain, mod Q), per_step consecutive polynomials to a step,
// to limb spectra [count / per_step][limbs][per_step][N/2]
void keys_to_fft_limbs_host(const host::NttTables& t, const uint64_t* keys_ntt, size_t count, uint32_t per_step,
                            const SplitPlan& plan, std::vector<double2>& out);
// GINX blind rotation with exact limb products (N = 1024 or 2048): one-bit (mb = 1, 2-4 digits,
// k.bskx the limbs of the BSK) or grouped mb = 2 (2-3 digits, k.bskx the limbs of the grouped
// keys [groups][limbs][3 subsets][2*digits][2][N/2]); the MV outputs are bit-identical to
// launch_blind_rotate's and left in the NTT domain
cudaError_t launch_blind_rotate_fft_split(const BlindRotateArgs& a, const FftKeyArgs& f, const SplitKeyArgs& k,
                                          const cbs_dmodulus* d_mod, uint32_t N, uint32_t batch, uint32_t mb,
                                          cudaStream_t s);

// mv_ntt: also transform the MV outputs to the NTT domain (the reference layout); false
// leaves them in the coefficient domain for the FFT HomTrace
cudaError_t launch_blind_rotate_fft(const BlindRotateArgs& a, const FftKeyArgs& f, const cbs_dmodulus* d_mod,
                                    uint32_t N, uint32_t batch, cudaStream_t s, bool mv_ntt = true);
// multi-bit form: groups of mb = 2 or 3 coefficients, f.bskf the grouped key spectra
// [ceil(n/mb)][2^mb - 1][2*digits][2][N/2]
cudaError_t launch_blind_rotate_fft_mb(const BlindRotateArgs& a, const FftKeyArgs& f, const cbs_dmodulus* d_mod,
                                       uint32_t N, uint32_t batch, uint32_t mb, cudaStream_t s, bool mv_ntt = true);
cudaError_t launch_trace_ss_fft(const TraceFftArgs& a, const FftKeyArgs& f, uint32_t N, uint32_t count, cudaStream_t s);
// digit spectra of the pair differences of `sets` fixed level-0 input sets (a.in, a.in_lut_stride,
// a.in_count, a.g, a.digits) into out [sets][in_count/2][2*digits][N/2]
cudaError_t launch_cmux_pair_spectra(const CmuxFftArgs& a, const FftKeyArgs& f, uint32_t N, uint32_t sets,
                                     double2* out, cudaStream_t s);
cudaError_t launch_cmux_level_fft(const CmuxFftArgs& a, const FftKeyArgs& f, uint32_t N, uint32_t luts,
                                  cudaStream_t s);
// spectra [polys][N/2] (slot-major) -> coefficient-domain polynomials [polys][N] mod Q, in place
cudaError_t launch_spectra_to_coef(double2* buf, uint64_t Q, const FftKeyArgs& f, uint32_t N, size_t polys,
                                   cudaStream_t s);
// coefficient-domain polynomials [polys][N] mod Q -> spectra [polys][N/2] (slot-major), out of place
cudaError_t launch_coef_to_spectra(const uint64_t* coef, double2* out, uint64_t Q, const FftKeyArgs& f, uint32_t N,
                                   size_t polys, cudaStream_t s);
DigitPrep make_digit_prep(uint64_t q, const Gadget& g, uint32_t digits);
// the FftTab<log2(N/2)> table (fft_core.cuh) computed in long double
void fft_tables_host(uint32_t N, std::vector<double2>& tab);
// in-place forward DIF transform of a (size M, twiddles w[e] = exp(2 pi i e / M), e < M/2) in
// long double: the host side of the key spectra
using cld = std::complex<long double>;
void host_dif(std::vector<cld>& a, const std::vector<cld>& w);
void keys_to_fft_host(const host::NttTables& t, const uint64_t* keys_ntt, size_t count, std::vector<double2>& out,
                      uint32_t split_bits = 0, uint32_t group = 0);
// key-column split of the HomTrace / SchemeSwitch key spectra: [row][k0_hi, k0_lo, k1][N/2]
constexpr uint32_t kTraceKeySplitBits = 27;

}  // namespace cbs
