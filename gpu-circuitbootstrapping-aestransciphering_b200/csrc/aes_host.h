// aes_host.h -- plaintext AES-128 pieces the transcipher needs on the host (key schedule,
// encryption T-tables), restating examples/aes_transcipher/aes128.cuh:99-121, :316-330
// from FIPS-197.
#pragma once

#include <array>
#include <cstdint>

namespace cbs {
namespace aes {

using Block = std::array<uint8_t, 16>;
using RoundKeys = std::array<Block, 11>;  // column-major state order (index = col*4 + row)

const std::array<uint8_t, 256>& sbox();
RoundKeys key_expand(const Block& key);
Block encrypt(const Block& in, const RoundKeys& rk);
// te[0..3] = Te0..Te3, te[4..7] = Te4_0..Te4_3 (final round)
std::array<std::array<uint32_t, 256>, 8> enc_tables();
inline uint32_t pack_be(uint8_t b0, uint8_t b1, uint8_t b2, uint8_t b3) {
    return (uint32_t(b0) << 24) | (uint32_t(b1) << 16) | (uint32_t(b2) << 8) | b3;
}

}  // namespace aes
}  // namespace cbs
