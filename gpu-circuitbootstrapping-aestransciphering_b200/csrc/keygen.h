// keygen.h -- seeded host key generation for the circuit-bootstrapping parameter set.
//
// Replaces the OpenFHE fork's KeyGen / RLWEKeyGen / CirBTKeyGen / KeySwitchGen
// (examples/aes_transcipher/main.cu:232-252) and the encrypted AES material
// (key_material.cuh:12-46, rlwe_tables.cuh:5-24).  Layouts are the device layouts of
// the reference (bitwise/src/cirbts/cirbts-init.cu:367-437; aes_gpu_ks.cuh:193-207):
//   bsk    [n][2*digits_g][2][N]  RGSW(s_i), NTT domain, row 2j+p carries m*g_j on poly p
//   ht     [rounds][digits_ht][2][N]  k1 - k0*s = -sigma_r(s) * g_j + e
//   ss     [digits_ss][2][N]          k1 - k0*s =  s^2 * g_j + e
//   ksk    [2][N][base_ks][n+1] u16   LWE_s(v * s'_i * base^j) mod qks
// RLWE ciphertexts are (a, b) with b - a*s = m + e; LWE (a, b) with b - <a,s> = m + e.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/cbs_b200.h"
#include "host_math.h"

namespace cbs {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed);
    uint64_t next();
    uint64_t uniform(uint64_t bound);  // [0, bound)
    double gaussian();                 // N(0, 1)
    int64_t rounded_gaussian(double sigma);
};

struct FastMod {
    uint64_t q, r0, r1;
    explicit FastMod(uint64_t q_);
    uint64_t mul(uint64_t a, uint64_t b) const;
    uint64_t add(uint64_t a, uint64_t b) const { uint64_t s = a + b; return s >= q ? s - q : s; }
    uint64_t sub(uint64_t a, uint64_t b) const { return a >= b ? a - b : a + q - b; }
    uint64_t from_signed(int64_t v) const;
};

struct HostKeys {
    std::vector<int32_t> s_lwe;   // n, binary
    std::vector<int32_t> s_rlwe;  // N, ternary
    std::vector<uint64_t> s_ntt;  // NTT(s_rlwe)
    std::vector<uint64_t> bsk, ht, ss;
    std::vector<uint16_t> ksk;
    std::vector<uint64_t> tv, gpow, gadd;
    std::vector<uint32_t> maps;
};

// Derived gadget powers of the RGSW output (AGPower of the reference, cirbts-init.cu:953-957)
std::vector<uint64_t> cbs_gadget_powers(const cbs_params& p);

void generate_keys(const cbs_params& p, const host::NttTables& t, uint64_t seed, HostKeys& k);
// gpow, tv, gadd and maps of k from the parameters (part of generate_keys; used alone when
// the evaluation keys come from the caller)
void derive_key_tables(const cbs_params& p, HostKeys& k);
// s_lwe (n), s_rlwe (N) and NTT(s_rlwe) of k from caller buffers
void set_secrets(const cbs_params& p, const host::NttTables& t, const int32_t* s_lwe, const int32_t* s_rlwe,
                 HostKeys& k);

// RLWE encryption of a coefficient-domain message (mod Q) into NTT-domain (a, b)
void rlwe_encrypt(const cbs_params& p, const host::NttTables& t, const HostKeys& k, Rng& rng,
                  const std::vector<uint64_t>& msg_coef, uint64_t* out_a_ntt, uint64_t* out_b_ntt);
// Multi-bit blind-rotation keys (the reference's CIRBTS_PBS_MULTIBIT = 2 / 3 / 4 grouping,
// bitwise/src/cirbts/cirbts-init.cu:376-565): LWE coefficients in groups of mb, and for every
// key subset S of a group (mb = 2, 3: every non-empty subset; mb = 4: the seven of
// coefficients 0-2 and {3}) an RGSW of prod_{i in S} s_i (0 for indices >= n), in the order of
// mb_subset_mask: out [ceil(n/mb)][mb_subsets(mb)][2*digits_g][2][N], NTT domain.
uint32_t mb_subsets(uint32_t mb);
uint32_t mb_subset_mask(uint32_t mb, uint32_t idx);
void generate_mb_bsk(const cbs_params& p, const host::NttTables& t, const HostKeys& k, uint32_t mb, uint64_t seed,
                     std::vector<uint64_t>& out);
// LMKCDEY keys (the reference's method = LMKCDEY, bitwise/src/cirbts/cirbts-init.cu:630-726;
// key set of cirbts-lmkcdey.cu:66-103): automorphism powers pows[0] = 2N - 5, then 5^i mod 2N
// (i = 1 .. num_auto_keys), or for window > 1 5^1 .. 5^window and 5^(2 window), 5^(3 window),
// ... below 5^(N/2); maps [count][N] the NTT-domain permutations out[t] = in[map[t]] of X -> X^k;
// eval [n][2*digits_g][2][N] = RGSW(X^{s_i}) and autok [count][digits_g][2][N] = RLWE(0) with
// b -= 2^{g (j+1)} psi_k(s), NTT domain, gadget powers 2^{g (j+1)} (the approximate
// decomposition drops the first g-bit digit).  One generator per key, seeded
// seed ^ (0x9e3779b97f4a7c15 (i + 1)) for eval key i and
// seed ^ 0x6c6d6b6364657921 ^ (0x9e3779b97f4a7c15 (k + 1)) for automorphism key k.
std::vector<uint32_t> lmkcdey_auto_pows(uint32_t N, uint32_t num_auto_keys, uint32_t window);
void lmkcdey_auto_maps(uint32_t N, uint32_t num_auto_keys, uint32_t window, std::vector<uint32_t>& maps);
void generate_lmkcdey_keys(const cbs_params& p, const host::NttTables& t, const HostKeys& k, uint32_t num_auto_keys,
                           uint32_t window, uint64_t seed, std::vector<uint64_t>& eval, std::vector<uint64_t>& autok);

// LWE encryption of m (already scaled) mod q under s_lwe
void lwe_encrypt(const cbs_params& p, const HostKeys& k, Rng& rng, uint64_t m, uint64_t* out_a, uint64_t* out_b);

}  // namespace cbs
