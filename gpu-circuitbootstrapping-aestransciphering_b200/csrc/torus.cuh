// torus.cuh -- shared pieces of the 32-bit-torus bootstrapping paths (gate bootstrap,
// torus circuit bootstrap): launch arguments of the FFT blind rotation and the key switch,
// and the host helpers for their keys.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "keygen.h"

namespace cbs {

// one request of a ragged batch: count ciphertexts a [count][n], b [count] in, outputs out_a,
// out_b; offset = number of ciphertexts in the requests before it
struct GateReq {
    const uint32_t* a;
    const uint32_t* b;
    uint32_t* out_a;
    uint32_t* out_b;
    uint32_t offset, count;
};

struct GateArgs {
    int gate;              // CBS_GATE_* or -1: bootstrap in1 as is
    const uint32_t* a1;    // [count][n]
    const uint32_t* b1;    // [count]
    const uint32_t* a2;
    const uint32_t* b2;
    uint32_t n, levels, bg_bits;
    const double2* bskf;   // [n][2*levels][2][M] key spectra, slot-major rows
    const double2* tab;    // FftTab<log2 M>
    void* ext;             // [items][N+1] extracted LWE (a then b), uint32 or uint64 torus
    const GateReq* reqs;   // ragged mode when non-null: items are the concatenated requests
    uint32_t num_reqs;
    uint32_t items;        // ciphertexts in total; CTAs loop over them with stride gridDim.x
    // test vectors: item i rotates the constant test vector mu[i % levels_tv] of input
    // i / levels_tv and adds b_add[i % levels_tv] to the extracted b (gates: one level, 1/8, 0)
    uint32_t levels_tv;
    uint64_t mu[8];        // in the kernel's torus width
    uint64_t b_add[8];
    // 32-bit torus only: a test vector [N] (coefficient domain) in place of the constant mu
    // (functional bootstrapping; levels_tv = 1)
    const uint32_t* tv;
    // 0 or 1: one coefficient per step (bskf [n][2*levels][2][M]); 2 or 3: groups of mb
    // coefficients (bskf [ceil(n/mb)][2^mb - 1][2*levels][2][M], the grouped kernel)
    uint32_t mb;
    // external-product arithmetic (CBS_FFT_*): 0 FP64 (bskf, tab); 1 split FP32, 2 FP32 (32-bit
    // torus, mb <= 1): bskf32 [n][2*levels][2][limbs][M] key-limb spectra, tab32 the FP32 table
    uint32_t fft_mode;
    const float2* bskf32;
    const float2* tab32;
};

cudaError_t gate_blind_rotate(const GateArgs& a, uint32_t N, uint32_t grid, cudaStream_t s);    // 32-bit torus
cudaError_t gate_blind_rotate64(const GateArgs& a, uint32_t N, uint32_t grid, cudaStream_t s);  // 64-bit torus
cudaError_t gate_keyswitch(const GateArgs& a, const uint32_t* ksk, uint32_t n, uint32_t N, uint32_t ks_bits,
                           uint32_t ks_levels, uint32_t* out_a, uint32_t* out_b, cudaStream_t s);

uint32_t torus_from_double(double x);
uint32_t torus_noise(Rng& rng, double sigma);
// b += a * z (negacyclic, z binary), mod 2^32
void mul_binary_acc(const uint32_t* a, const int32_t* z, uint32_t N, uint32_t* b);
// torus32 key polynomials [count][N] -> FFT spectra [count][N/2] in the slot-major order of
// the blind-rotation kernels
void torus_keys_to_fft(uint32_t N, const uint32_t* keys, size_t count, std::vector<double2>& out);
void torus_keys_to_fft(uint32_t N, const uint64_t* keys, size_t count, std::vector<double2>& out);
// FP32 form: each torus32 polynomial as `limbs` spectra [count][limbs][N/2]; limbs = 2 splits
// k = lo + 2^S hi, S = log2 N + 14, with lo the signed S-bit residue and hi the signed
// (32 - S)-bit rest; limbs = 1 keeps the centred k
void torus_keys_to_fft32(uint32_t N, const uint32_t* keys, size_t count, uint32_t limbs, std::vector<float2>& out);

}  // namespace cbs
