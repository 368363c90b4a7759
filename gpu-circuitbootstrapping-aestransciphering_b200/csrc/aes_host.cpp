// aes_host.cpp -- see aes_host.h.
#include "aes_host.h"

namespace cbs {
namespace aes {

static uint8_t gf_mul(uint8_t a, uint8_t b) {
    uint8_t p = 0;
    while (b) {
        if (b & 1) p ^= a;
        a = static_cast<uint8_t>((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
        b >>= 1;
    }
    return p;
}

const std::array<uint8_t, 256>& sbox() {
    static const std::array<uint8_t, 256> table = [] {
        std::array<uint8_t, 256> s{};
        for (int x = 0; x < 256; ++x) {
            uint8_t inv = 0;
            for (int y = 1; x && y < 256; ++y)
                if (gf_mul(static_cast<uint8_t>(x), static_cast<uint8_t>(y)) == 1) {
                    inv = static_cast<uint8_t>(y);
                    break;
                }
            uint8_t v = inv;
            for (int i = 1; i <= 4; ++i) v ^= static_cast<uint8_t>((inv << i) | (inv >> (8 - i)));
            s[x] = static_cast<uint8_t>(v ^ 0x63);
        }
        return s;
    }();
    return table;
}

RoundKeys key_expand(const Block& key) {
    const auto& sb = sbox();
    static const uint8_t rcon[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
    uint8_t w[44][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) w[i][j] = key[4 * i + j];
    for (int i = 4; i < 44; ++i) {
        uint8_t t[4] = {w[i - 1][0], w[i - 1][1], w[i - 1][2], w[i - 1][3]};
        if (i % 4 == 0) {
            const uint8_t t0 = t[0];
            t[0] = static_cast<uint8_t>(sb[t[1]] ^ rcon[i / 4 - 1]);
            t[1] = sb[t[2]];
            t[2] = sb[t[3]];
            t[3] = sb[t0];
        }
        for (int j = 0; j < 4; ++j) w[i][j] = static_cast<uint8_t>(w[i - 4][j] ^ t[j]);
    }
    RoundKeys rk{};
    for (int r = 0; r < 11; ++r)
        for (int c = 0; c < 4; ++c)
            for (int row = 0; row < 4; ++row) rk[r][c * 4 + row] = w[r * 4 + c][row];
    return rk;
}

Block encrypt(const Block& in, const RoundKeys& rk) {
    const auto& sb = sbox();
    Block s{}, t{};
    for (int i = 0; i < 16; ++i) s[i] = in[i] ^ rk[0][i];
    for (int r = 1; r <= 10; ++r) {
        for (auto& v : s) v = sb[v];
        for (int row = 0; row < 4; ++row)
            for (int c = 0; c < 4; ++c) t[c * 4 + row] = s[((c + row) & 3) * 4 + row];
        s = t;
        if (r != 10) {
            for (int c = 0; c < 4; ++c) {
                const uint8_t a0 = s[c * 4], a1 = s[c * 4 + 1], a2 = s[c * 4 + 2], a3 = s[c * 4 + 3];
                s[c * 4 + 0] = static_cast<uint8_t>(gf_mul(a0, 2) ^ gf_mul(a1, 3) ^ a2 ^ a3);
                s[c * 4 + 1] = static_cast<uint8_t>(a0 ^ gf_mul(a1, 2) ^ gf_mul(a2, 3) ^ a3);
                s[c * 4 + 2] = static_cast<uint8_t>(a0 ^ a1 ^ gf_mul(a2, 2) ^ gf_mul(a3, 3));
                s[c * 4 + 3] = static_cast<uint8_t>(gf_mul(a0, 3) ^ a1 ^ a2 ^ gf_mul(a3, 2));
            }
        }
        for (int i = 0; i < 16; ++i) s[i] ^= rk[r][i];
    }
    return s;
}

std::array<std::array<uint32_t, 256>, 8> enc_tables() {
    const auto& sb = sbox();
    std::array<std::array<uint32_t, 256>, 8> te{};
    for (int x = 0; x < 256; ++x) {
        const uint8_t s = sb[x];
        const uint32_t t0 = pack_be(gf_mul(s, 2), s, s, gf_mul(s, 3));
        te[0][x] = t0;
        te[1][x] = (t0 >> 8) | (t0 << 24);
        te[2][x] = (t0 >> 16) | (t0 << 16);
        te[3][x] = (t0 >> 24) | (t0 << 8);
        te[4][x] = pack_be(s, 0, 0, 0);
        te[5][x] = pack_be(0, s, 0, 0);
        te[6][x] = pack_be(0, 0, s, 0);
        te[7][x] = pack_be(0, 0, 0, s);
    }
    return te;
}

}  // namespace aes
}  // namespace cbs
