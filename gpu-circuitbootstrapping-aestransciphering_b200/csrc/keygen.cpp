// keygen.cpp -- see keygen.h.
#include "keygen.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <thread>

namespace cbs {

using u128 = unsigned __int128;

// ---- RNG: xoshiro256** seeded through splitmix64 ----
static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

Rng::Rng(uint64_t seed) {
    uint64_t x = seed;
    for (auto& w : s) w = splitmix(x);
}

uint64_t Rng::next() {
    const uint64_t r = ((s[1] * 5) << 7 | (s[1] * 5) >> 57) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
    return r;
}

uint64_t Rng::uniform(uint64_t bound) {
    // rejection sampling on the top bits: exact uniform
    int bits = 0;
    while (bits < 64 && (bound - 1) >> bits) ++bits;
    const uint64_t mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    for (;;) {
        const uint64_t v = next() & mask;
        if (v < bound) return v;
    }
}

double Rng::gaussian() {
    // Box-Muller
    const double u1 = (static_cast<double>(next() >> 11) + 1.0) * 0x1.0p-53;
    const double u2 = static_cast<double>(next() >> 11) * 0x1.0p-53;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
}

int64_t Rng::rounded_gaussian(double sigma) { return static_cast<int64_t>(std::llround(gaussian() * sigma)); }

// ---- fast host modular multiply (Barrett with floor(2^128 / q)) ----
FastMod::FastMod(uint64_t q_) : q(q_) { host::barrett_ratio(q_, r0, r1); }

uint64_t FastMod::mul(uint64_t a, uint64_t b) const {
    const u128 x = u128(a) * b;
    const uint64_t xlo = static_cast<uint64_t>(x), xhi = static_cast<uint64_t>(x >> 64);
    const u128 p0 = u128(xlo) * r0, p1 = u128(xlo) * r1, p2 = u128(xhi) * r0;
    const u128 mid = (p0 >> 64) + static_cast<uint64_t>(p1) + static_cast<uint64_t>(p2);
    const uint64_t quot = xhi * r1 + static_cast<uint64_t>(p1 >> 64) + static_cast<uint64_t>(p2 >> 64) +
                          static_cast<uint64_t>(mid >> 64);
    uint64_t r = xlo - quot * q;
    while (r >= q) r -= q;
    return r;
}

uint64_t FastMod::from_signed(int64_t v) const {
    const int64_t m = v % static_cast<int64_t>(q);
    return m < 0 ? static_cast<uint64_t>(m + static_cast<int64_t>(q)) : static_cast<uint64_t>(m);
}

// fast host NTT with Shoup twiddles (same transform as host::ntt_forward_host)
static void ntt_fwd_fast(uint64_t* a, const host::NttTables& t) {
    const uint32_t n = t.n;
    const uint64_t q = t.q;
    for (uint32_t m = 1; m < n; m <<= 1) {
        const uint32_t h = n / (2 * m);
        for (uint32_t k = 0; k < m; ++k) {
            const uint64_t w = t.rp[m + k], ws = t.rp_sh[m + k];
            for (uint32_t j = 2 * k * h; j < 2 * k * h + h; ++j) {
                const uint64_t y = a[j + h];
                const uint64_t hi = static_cast<uint64_t>((u128(y) * ws) >> 64);
                uint64_t v = y * w - hi * q;
                if (v >= q) v -= q;
                const uint64_t u = a[j];
                uint64_t s = u + v;
                if (s >= q) s -= q;
                a[j] = s;
                a[j + h] = u >= v ? u - v : u + q - v;
            }
        }
    }
}

std::vector<uint64_t> cbs_gadget_powers(const cbs_params& p) {
    int gb = 0;
    while ((1u << gb) < p.base_cc) ++gb;
    int logq = 0;
    while (logq < 64 && (p.Q >> logq)) ++logq;
    int ign = logq - static_cast<int>(p.num_lut) * gb;
    if (ign < 0) ign = 0;
    std::vector<uint64_t> g(p.num_lut);
    for (uint32_t j = 0; j < p.num_lut; ++j) g[j] = 1ull << (ign + static_cast<int>(j) * gb);
    return g;
}

static std::vector<uint64_t> gadget_of(uint64_t Q, uint32_t base, uint32_t digits) {
    int gb = 0;
    while ((1u << gb) < base) ++gb;
    int logq = 0;
    while (logq < 64 && (Q >> logq)) ++logq;
    int ign = logq - static_cast<int>(digits) * gb;
    if (ign < 0) ign = 0;
    std::vector<uint64_t> g(digits);
    for (uint32_t j = 0; j < digits; ++j) g[j] = (1ull << (ign + static_cast<int>(j) * gb)) % Q;
    return g;
}

// one fresh RLWE sample of zero: a uniform in the NTT domain, b = a*s + NTT(e)
static void rlwe_zero(const cbs_params& p, const host::NttTables& t, const HostKeys& k, const FastMod& fm, Rng& rng,
                      uint64_t* a, uint64_t* b, std::vector<uint64_t>& tmp) {
    const uint32_t N = p.N;
    for (uint32_t i = 0; i < N; ++i) a[i] = rng.uniform(p.Q);
    tmp.resize(N);
    for (uint32_t i = 0; i < N; ++i) tmp[i] = fm.from_signed(rng.rounded_gaussian(p.sigma_rlwe));
    ntt_fwd_fast(tmp.data(), t);
    for (uint32_t i = 0; i < N; ++i) b[i] = fm.add(fm.mul(a[i], k.s_ntt[i]), tmp[i]);
}

void rlwe_encrypt(const cbs_params& p, const host::NttTables& t, const HostKeys& k, Rng& rng,
                  const std::vector<uint64_t>& msg_coef, uint64_t* out_a, uint64_t* out_b) {
    FastMod fm(p.Q);
    std::vector<uint64_t> tmp;
    rlwe_zero(p, t, k, fm, rng, out_a, out_b, tmp);
    std::vector<uint64_t> m(msg_coef);
    ntt_fwd_fast(m.data(), t);
    for (uint32_t i = 0; i < p.N; ++i) out_b[i] = fm.add(out_b[i], m[i]);
}

uint32_t mb_subsets(uint32_t mb) { return mb == 4 ? 8u : (1u << mb) - 1u; }

uint32_t mb_subset_mask(uint32_t mb, uint32_t idx) {
    // subsets of {0..mb-1} ordered by size, then lexicographically: for mb = 3,
    // {0} {1} {2} {0,1} {0,2} {1,2} {0,1,2} (the reference's k0 k1 k2 k01 k02 k12 k012,
    // cirbts-init.cu:499-530); for mb = 2, {0} {1} {0,1} (k0 k1 k01, :485-498).  mb = 4 is the
    // reference's staged grouping (:536-565): k0 k1 k2 k3 k01 k02 k12 k012, the mb = 3 keys of
    // coefficients 0-2 and the one-bit key of coefficient 3.
    static const uint32_t order2[3] = {0b01, 0b10, 0b11};
    static const uint32_t order3[7] = {0b001, 0b010, 0b100, 0b011, 0b101, 0b110, 0b111};
    static const uint32_t order4[8] = {0b0001, 0b0010, 0b0100, 0b1000, 0b0011, 0b0101, 0b0110, 0b0111};
    if (mb == 1) return 1u;
    if (mb == 2) return order2[idx];
    if (mb == 4) return order4[idx];
    return order3[idx];
}

void generate_mb_bsk(const cbs_params& p, const host::NttTables& t, const HostKeys& k, uint32_t mb, uint64_t seed,
                     std::vector<uint64_t>& out) {
    const uint32_t N = p.N, n = p.n, l2 = 2 * p.digits_g, K = mb_subsets(mb);
    const uint32_t groups = (n + mb - 1) / mb;
    const uint64_t Q = p.Q;
    FastMod fm(Q);
    const auto gbr = gadget_of(Q, p.base_g, p.digits_g);
    out.assign(static_cast<size_t>(groups) * K * l2 * 2 * N, 0);
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th) {
        pool.emplace_back([&, th] {
            std::vector<uint64_t> tmp;
            for (uint32_t g = th; g < groups; g += nth) {
                // one generator per group, so the keys do not depend on the thread count
                Rng rng(seed ^ (0x9e3779b97f4a7c15ull * (g + 1)));
                for (uint32_t kk = 0; kk < K; ++kk) {
                    const uint32_t mask = mb_subset_mask(mb, kk);
                    uint32_t prod = 1;  // the product of the subset's secret bits (0 past n)
                    for (uint32_t i = 0; i < mb; ++i)
                        if (mask & (1u << i)) {
                            const uint32_t idx = g * mb + i;
                            prod &= (idx < n) ? static_cast<uint32_t>(k.s_lwe[idx]) : 0u;
                        }
                    for (uint32_t r = 0; r < l2; ++r) {
                        uint64_t* a = out.data() + ((static_cast<size_t>(g) * K + kk) * l2 + r) * 2 * N;
                        uint64_t* b = a + N;
                        rlwe_zero(p, t, k, fm, rng, a, b, tmp);
                        if (prod) {
                            const uint64_t m = gbr[r >> 1];
                            uint64_t* tgt = (r & 1) ? b : a;
                            for (uint32_t c = 0; c < N; ++c) tgt[c] = fm.add(tgt[c], m);
                        }
                    }
                }
            }
        });
    }
    for (auto& th : pool) th.join();
}

std::vector<uint32_t> lmkcdey_auto_pows(uint32_t N, uint32_t num_auto_keys, uint32_t window) {
    const uint32_t M = 2 * N;
    auto pow5 = [M](uint32_t k) {
        uint64_t v = 1;
        for (uint32_t i = 0; i < k; ++i) v = (v * 5) % M;
        return static_cast<uint32_t>(v);
    };
    std::vector<uint32_t> pows{M - 5};
    if (window > 1) {
        for (uint32_t k = 1; k <= window; ++k) pows.push_back(pow5(k));
        for (uint32_t k = 2 * window; k <= N / 2 - 1; k += window) pows.push_back(pow5(k));
    } else {
        for (uint32_t k = 1; k <= num_auto_keys; ++k) pows.push_back(pow5(k));
    }
    return pows;
}

void lmkcdey_auto_maps(uint32_t N, uint32_t num_auto_keys, uint32_t window, std::vector<uint32_t>& maps) {
    uint32_t logn = 0;
    while ((1u << logn) < N) ++logn;
    auto brev = [logn](uint32_t x) {
        uint32_t r = 0;
        for (uint32_t i = 0; i < logn; ++i) r |= ((x >> i) & 1u) << (logn - 1 - i);
        return r;
    };
    const auto pows = lmkcdey_auto_pows(N, num_auto_keys, window);
    maps.assign(pows.size() * N, 0);
    // slot t holds the evaluation at zeta^(2 brev(t) + 1); psi_k reads the slot of its k-th power
    for (size_t k = 0; k < pows.size(); ++k)
        for (uint32_t t = 0; t < N; ++t) {
            const uint64_t e = 2ull * brev(t) + 1;
            maps[k * N + t] = brev(static_cast<uint32_t>(((e * pows[k]) & (2ull * N - 1)) >> 1));
        }
}

void generate_lmkcdey_keys(const cbs_params& p, const host::NttTables& t, const HostKeys& k, uint32_t num_auto_keys,
                           uint32_t window, uint64_t seed, std::vector<uint64_t>& eval, std::vector<uint64_t>& autok) {
    const uint32_t N = p.N, n = p.n, dg = p.digits_g, M = 2 * N;
    int g = 0;
    while ((1u << g) < p.base_g) ++g;
    const uint64_t Q = p.Q;
    FastMod fm(Q);
    std::vector<uint64_t> gp(dg);
    for (uint32_t j = 0; j < dg; ++j) gp[j] = (1ull << (g * (j + 1))) % Q;
    std::vector<uint32_t> maps;
    lmkcdey_auto_maps(N, num_auto_keys, window, maps);
    const uint32_t count = static_cast<uint32_t>(maps.size() / N);
    eval.assign(static_cast<size_t>(n) * 2 * dg * 2 * N, 0);
    autok.assign(static_cast<size_t>(count) * dg * 2 * N, 0);
    const unsigned nth = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned th = 0; th < nth; ++th) {
        pool.emplace_back([&, th] {
            std::vector<uint64_t> tmp, mono(N);
            for (uint32_t i = th; i < n; i += nth) {
                Rng rng(seed ^ (0x9e3779b97f4a7c15ull * (i + 1)));
                const int64_t e = ((static_cast<int64_t>(k.s_lwe[i]) % M) + M) % M;
                std::fill(mono.begin(), mono.end(), 0);
                if (e < N) mono[e] = 1 % Q;
                else mono[e - N] = Q - 1;
                ntt_fwd_fast(mono.data(), t);
                for (uint32_t r = 0; r < 2 * dg; ++r) {
                    uint64_t* a = eval.data() + (static_cast<size_t>(i) * 2 * dg + r) * 2 * N;
                    uint64_t* b = a + N;
                    rlwe_zero(p, t, k, fm, rng, a, b, tmp);
                    uint64_t* tgt = (r & 1) ? b : a;
                    for (uint32_t c = 0; c < N; ++c) tgt[c] = fm.add(tgt[c], fm.mul(mono[c], gp[r >> 1]));
                }
            }
            for (uint32_t kk = th; kk < count; kk += nth) {
                Rng rng(seed ^ 0x6c6d6b6364657921ull ^ (0x9e3779b97f4a7c15ull * (kk + 1)));
                const uint32_t* map = maps.data() + static_cast<size_t>(kk) * N;
                for (uint32_t j = 0; j < dg; ++j) {
                    uint64_t* a = autok.data() + (static_cast<size_t>(kk) * dg + j) * 2 * N;
                    uint64_t* b = a + N;
                    rlwe_zero(p, t, k, fm, rng, a, b, tmp);
                    for (uint32_t c = 0; c < N; ++c) b[c] = fm.sub(b[c], fm.mul(k.s_ntt[map[c]], gp[j]));
                }
            }
        });
    }
    for (auto& th : pool) th.join();
}

void lwe_encrypt(const cbs_params& p, const HostKeys& k, Rng& rng, uint64_t m, uint64_t* out_a, uint64_t* out_b) {
    const uint64_t q = p.q_lwe;
    u128 acc = 0;
    for (uint32_t i = 0; i < p.n; ++i) {
        out_a[i] = rng.uniform(q);
        if (k.s_lwe[i]) acc += out_a[i];
    }
    const int64_t e = rng.rounded_gaussian(p.sigma_lwe);
    const int64_t qi = static_cast<int64_t>(q);
    int64_t bm = static_cast<int64_t>((acc + m) % q) + (e % qi);
    bm %= qi;
    if (bm < 0) bm += qi;
    *out_b = static_cast<uint64_t>(bm);
}

// The material a context derives from the parameters alone: the gadget powers, the
// multi-value test vector, the finalize constants and the NTT-domain automorphism maps.
void derive_key_tables(const cbs_params& p, HostKeys& k) {
    const uint32_t N = p.N;
    const uint64_t Q = p.Q;
    FastMod fm(Q);
    const uint32_t logn = static_cast<uint32_t>(__builtin_ctz(N));
    const uint32_t rounds = logn - p.trace_shift;
    // test vector: slot j of each 2^bw block holds -+g_j/2 (negative on the first half)
    k.gpow = cbs_gadget_powers(p);
    uint32_t bw = 0;
    while ((1u << bw) < p.num_lut) ++bw;
    k.tv.assign(N, 0);
    for (uint32_t i = 0; i < N; ++i) {
        const uint32_t slot = i & ((1u << bw) - 1);
        if (slot >= p.num_lut) continue;
        const uint64_t half = (k.gpow[slot] >> 1) % Q;
        k.tv[i] = (i < N / 2) ? (half ? Q - half : 0) : half;
    }
    const uint64_t ninv = host::invmod(N, Q);
    k.gadd.resize(p.num_lut);
    for (uint32_t j = 0; j < p.num_lut; ++j) k.gadd[j] = fm.mul((k.gpow[j] >> 1) % Q, ninv);

    // NTT-domain automorphism maps (kernel.cu:7554-7571)
    k.maps.assign(static_cast<size_t>(rounds) * N, 0);
    for (uint32_t lv = 0; lv < rounds; ++lv) {
        const uint64_t kk = (static_cast<uint64_t>(N) >> lv) + 1;
        for (uint32_t tid = 0; tid < N; ++tid) {
            const uint32_t j = host::bit_reverse(tid, static_cast<int>(logn));
            const uint32_t idx = static_cast<uint32_t>((((2ull * j + 1) * kk) & (2ull * N - 1)) >> 1);
            k.maps[static_cast<size_t>(lv) * N + tid] = host::bit_reverse(idx, static_cast<int>(logn));
        }
    }
}

void set_secrets(const cbs_params& p, const host::NttTables& t, const int32_t* s_lwe, const int32_t* s_rlwe,
                 HostKeys& k) {
    FastMod fm(p.Q);
    k.s_lwe.assign(s_lwe, s_lwe + p.n);
    k.s_rlwe.assign(s_rlwe, s_rlwe + p.N);
    k.s_ntt.resize(p.N);
    for (uint32_t i = 0; i < p.N; ++i) k.s_ntt[i] = fm.from_signed(k.s_rlwe[i]);
    ntt_fwd_fast(k.s_ntt.data(), t);
}

void generate_keys(const cbs_params& p, const host::NttTables& t, uint64_t seed, HostKeys& k) {
    const uint32_t N = p.N, n = p.n;
    const uint64_t Q = p.Q;
    FastMod fm(Q);
    Rng rng(seed);
    std::vector<uint64_t> tmp;

    // secrets: binary LWE key, ternary RLWE key
    k.s_lwe.resize(n);
    for (auto& v : k.s_lwe) v = static_cast<int32_t>(rng.next() & 1);
    k.s_rlwe.resize(N);
    for (auto& v : k.s_rlwe) v = static_cast<int32_t>(rng.uniform(3)) - 1;
    k.s_ntt.resize(N);
    for (uint32_t i = 0; i < N; ++i) k.s_ntt[i] = fm.from_signed(k.s_rlwe[i]);
    ntt_fwd_fast(k.s_ntt.data(), t);

    // bootstrapping key: RGSW(s_i), rows r = 2j + poly carry s_i * g_j on component poly
    const uint32_t l2 = 2 * p.digits_g;
    const auto gbr = gadget_of(Q, p.base_g, p.digits_g);
    k.bsk.assign(static_cast<size_t>(n) * l2 * 2 * N, 0);
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t r = 0; r < l2; ++r) {
            uint64_t* a = k.bsk.data() + (static_cast<size_t>(i) * l2 + r) * 2 * N;
            uint64_t* b = a + N;
            rlwe_zero(p, t, k, fm, rng, a, b, tmp);
            if (k.s_lwe[i]) {
                const uint64_t m = gbr[r >> 1];
                uint64_t* tgt = (r & 1) ? b : a;
                for (uint32_t c = 0; c < N; ++c) tgt[c] = fm.add(tgt[c], m);
            }
        }
    }

    // HomTrace keys: k1 - k0*s = -sigma_r(s) * g_j + e, automorphism X -> X^(N/2^r + 1)
    const uint32_t logn = static_cast<uint32_t>(__builtin_ctz(N));
    const uint32_t rounds = logn - p.trace_shift;
    const auto ght = gadget_of(Q, p.base_ht, p.digits_ht);
    k.ht.assign(static_cast<size_t>(rounds) * p.digits_ht * 2 * N, 0);
    std::vector<uint64_t> sig(N);
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint64_t kk = (static_cast<uint64_t>(N) >> r) + 1;
        std::fill(sig.begin(), sig.end(), 0);
        for (uint32_t i = 0; i < N; ++i) {
            const uint64_t e = (static_cast<uint64_t>(i) * kk) % (2ull * N);
            const int64_t v = k.s_rlwe[i];
            if (e < N) sig[e] = fm.add(sig[e], fm.from_signed(v));
            else sig[e - N] = fm.add(sig[e - N], fm.from_signed(-v));
        }
        ntt_fwd_fast(sig.data(), t);
        for (uint32_t j = 0; j < p.digits_ht; ++j) {
            uint64_t* a = k.ht.data() + (static_cast<size_t>(r) * p.digits_ht + j) * 2 * N;
            uint64_t* b = a + N;
            rlwe_zero(p, t, k, fm, rng, a, b, tmp);
            for (uint32_t c = 0; c < N; ++c) b[c] = fm.sub(b[c], fm.mul(sig[c], ght[j]));
        }
    }

    // SchemeSwitch key: k1 - k0*s = s^2 * g_j + e
    const auto gss = gadget_of(Q, p.base_ss, p.digits_ss);
    k.ss.assign(static_cast<size_t>(p.digits_ss) * 2 * N, 0);
    for (uint32_t j = 0; j < p.digits_ss; ++j) {
        uint64_t* a = k.ss.data() + static_cast<size_t>(j) * 2 * N;
        uint64_t* b = a + N;
        rlwe_zero(p, t, k, fm, rng, a, b, tmp);
        for (uint32_t c = 0; c < N; ++c) b[c] = fm.add(b[c], fm.mul(fm.mul(k.s_ntt[c], k.s_ntt[c]), gss[j]));
    }

    derive_key_tables(p, k);

    // extraction key switch N -> n: LWE_s(v * s'_i * B^j) mod qks, u16 packed
    const uint32_t qks = p.qks, bks = p.base_ks, outlen = n + 1;
    const uint32_t mask = qks - 1;
    k.ksk.assign(static_cast<size_t>(2) * N * bks * outlen, 0);
    for (uint32_t j = 0; j < 2; ++j) {
        const uint32_t bj = (j == 0) ? 1u : bks;
        for (uint32_t i = 0; i < N; ++i) {
            const uint32_t si = static_cast<uint32_t>(k.s_rlwe[i] + static_cast<int32_t>(qks)) & mask;
            for (uint32_t v = 0; v < bks; ++v) {
                uint16_t* row = k.ksk.data() + ((static_cast<size_t>(j) * N + i) * bks + v) * outlen;
                uint32_t acc = 0;
                for (uint32_t c = 0; c < n; ++c) {
                    const uint32_t a = static_cast<uint32_t>(rng.next() & mask);
                    row[c] = static_cast<uint16_t>(a);
                    if (k.s_lwe[c]) acc += a;
                }
                const int64_t e = rng.rounded_gaussian(p.sigma_lwe);
                const uint32_t m = (v * si * bj) & mask;
                row[n] = static_cast<uint16_t>((acc + m + static_cast<uint32_t>(e)) & mask);
            }
        }
    }
}

}  // namespace cbs
