// fft_kernels.cuh -- FP64 FFT blind-rotation backend: launch interface and host key prep.
#pragma once

#include <cuda_runtime.h>

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

cudaError_t launch_blind_rotate_fft(const BlindRotateArgs& a, const FftKeyArgs& f, const cbs_dmodulus* d_mod,
                                    uint32_t N, uint32_t batch, cudaStream_t s);
// the FftTab<log2(N/2)> table (fft_core.cuh) computed in long double
void fft_tables_host(uint32_t N, std::vector<double2>& tab);
void keys_to_fft_host(const host::NttTables& t, const uint64_t* keys_ntt, size_t count, std::vector<double2>& out);

}  // namespace cbs
