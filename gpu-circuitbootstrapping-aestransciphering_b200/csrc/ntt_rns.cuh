// ntt_rns.cuh -- multi-prime (RNS) negacyclic NTT for N = 2^10 .. 2^17.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace cbs {

// Tables of every prime of a modulus chain, Phantom's DNTTTable layout (include/ntt.cuh:100-160):
// tw/tws/itw/itws are [primes][N] (bit-reversed root powers, Shoup quotients; n^-1 folded into
// itw[1]); q, n_inv, n_inv_s are [primes].  limb_prime[l] is the table row used by limb l of the
// data, so one launch can cover any subset of the chain (Ql, P, Ql+P, the complement of a digit).
struct RnsNttArgs {
    const uint64_t* tw = nullptr;
    const uint64_t* tws = nullptr;
    const uint64_t* itw = nullptr;
    const uint64_t* itws = nullptr;
    const uint64_t* q = nullptr;
    const uint64_t* n_inv = nullptr;
    const uint64_t* n_inv_s = nullptr;
    // the tw / itw tables as doubles, set only when every prime is below 2^50: the 2-D
    // transforms (N >= 2^13) then run on the FP64 pipe, with the same results
    const double* twd = nullptr;
    const double* itwd = nullptr;
    uint32_t* fault = nullptr;  // device word: bit 1 set if a bulk copy's bounded wait expired
    const uint32_t* limb_prime = nullptr;  // device [limbs]: table row of launch limb l
    const uint32_t* limb_slot = nullptr;   // device [limbs]: limb position in the polynomial (null: l)
    uint32_t limbs = 0;
    uint64_t poly_stride = 0;  // words between polynomials
    // out of place: the first phase reads from in (same limb slots, in_poly_stride) when non-null
    const uint64_t* in = nullptr;
    uint64_t in_poly_stride = 0;
    // inverse only: outputs multiplied by scale[l] (Shoup scale_s[l]) when non-null
    const uint64_t* scale = nullptr;
    const uint64_t* scale_s = nullptr;
    // forward only, fused moddown epilogue (src/ntt/ntt_moddown.cu:222): with v the NTT output
    // of launch limb l of poly p, epi = 1 writes dst = (cx - v) * f[l], epi = 2 adds it to dst;
    // cx limb l of poly p at epi_cx + p * epi_cx_stride + l * N, dst likewise; data is left
    // in its lazy intermediate state.
    int epi = 0;
    const uint64_t* epi_cx = nullptr;
    uint64_t* epi_dst = nullptr;
    uint64_t epi_cx_stride = 0, epi_dst_stride = 0;
    const uint64_t* epi_f = nullptr;
    const uint64_t* epi_fs = nullptr;
};

// Launch limb l of poly p lives at data + p * poly_stride + slot(l) * N; in place.
// Forward: coefficient -> NTT domain (bit-reversed), outputs in [0, q).  Inverse: the reverse,
// n^-1 applied, outputs in [0, q).
cudaError_t rns_ntt(uint64_t* data, const RnsNttArgs& a, uint32_t log_n, size_t polys, bool inverse,
                    cudaStream_t s);

}  // namespace cbs
