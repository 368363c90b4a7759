// ref_shim.cpp -- extern "C" wrappers around the reference's own host code, compiled
// from the reference sources in place (recipe: oracle/Makefile, target ref).  TEST
// INFRASTRUCTURE ONLY: used to pin the oracle (tests/, tests/golden/make_golden.py) and
// as the reference-kind CPU baseline.  No reference source is copied into this
// repository; the reference headers are included from the reference tree at build time.
#include <array>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "host/ntt.h"
#include "host/numth.h"

namespace refaes {
// Plain AES-128 and T-table builders from examples/aes_transcipher/aes128.cuh.
#include "aes128.cuh"
}  // namespace refaes

extern "C" {

// src/host/numth.cu:207 get_primes
int ref_get_primes(uint32_t ntt_size, int bit_size, uint32_t count, uint64_t* out) {
    try {
        auto v = phantom::arith::get_primes(ntt_size, bit_size, count);
        for (uint32_t i = 0; i < count; ++i) out[i] = v[i].value();
        return 0;
    } catch (...) {
        return -1;
    }
}

// src/host/ntt.cu:11 NTT tables
int ref_ntt_tables(uint32_t log_n, uint64_t q, uint64_t* rp, uint64_t* rp_sh, uint64_t* irp, uint64_t* irp_sh,
                   uint64_t* n_inv) {
    try {
        phantom::arith::Modulus m(q);
        phantom::arith::NTT t(static_cast<int>(log_n), m);
        const size_t n = size_t(1) << log_n;
        std::memcpy(rp, t.get_from_root_powers().data(), n * 8);
        std::memcpy(rp_sh, t.get_from_root_powers_shoup().data(), n * 8);
        std::memcpy(irp, t.get_from_inv_root_powers().data(), n * 8);
        std::memcpy(irp_sh, t.get_from_inv_root_powers_shoup().data(), n * 8);
        n_inv[0] = t.inv_degree_modulo();
        n_inv[1] = t.inv_degree_modulo_shoup();
        return 0;
    } catch (...) {
        return -1;
    }
}

// Barrett constant of src/host/modulus.h (const_ratio[0..1]) for DModulus parity
int ref_modulus_ratio(uint64_t q, uint64_t* ratio2) {
    phantom::arith::Modulus m(q);
    ratio2[0] = m.const_ratio()[0];
    ratio2[1] = m.const_ratio()[1];
    return 0;
}

// aes128.cuh:151 Aes128EncryptPlain after Aes128KeyExpand
void ref_aes128_encrypt(const uint8_t* key, const uint8_t* in, uint8_t* out) {
    std::array<uint8_t, 16> k{}, p{};
    std::memcpy(k.data(), key, 16);
    std::memcpy(p.data(), in, 16);
    const auto rk = refaes::Aes128KeyExpand(k);
    const auto c = refaes::Aes128EncryptPlain(p, rk);
    std::memcpy(out, c.data(), 16);
}

// aes128.cuh:316 BuildAesEncTables -> te[8][256]
void ref_aes_enc_tables(uint32_t* te) {
    const auto t = refaes::BuildAesEncTables();
    const refaes::Table256* tabs[8] = {&t.te0, &t.te1, &t.te2, &t.te3, &t.te4_0, &t.te4_1, &t.te4_2, &t.te4_3};
    for (int i = 0; i < 8; ++i) std::memcpy(te + 256 * i, tabs[i]->data(), 256 * 4);
}

// aes128.cuh:99 Aes128KeyExpand -> rk[11][16]
void ref_aes128_key_expand(const uint8_t* key, uint8_t* rk) {
    std::array<uint8_t, 16> k{};
    std::memcpy(k.data(), key, 16);
    const auto r = refaes::Aes128KeyExpand(k);
    for (int i = 0; i < 11; ++i) std::memcpy(rk + 16 * i, r[i].data(), 16);
}
}
