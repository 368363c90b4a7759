// host_math.cpp -- see host_math.h.
#include "host_math.h"

namespace cbs {
namespace host {

using u128 = unsigned __int128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return static_cast<uint64_t>((u128(a) * b) % q); }

uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = mulmod(r, a, q);
        a = mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}

uint64_t invmod(uint64_t a, uint64_t q) {
    __int128 t = 0, nt = 1, r = q, nr = a % q;
    while (nr != 0) {
        const __int128 quo = r / nr;
        __int128 tmp = t - quo * nt;
        t = nt;
        nt = tmp;
        tmp = r - quo * nr;
        r = nr;
        nr = tmp;
    }
    if (r != 1) return 0;
    if (t < 0) t += q;
    return static_cast<uint64_t>(t);
}

uint64_t shoup(uint64_t w, uint64_t q) { return static_cast<uint64_t>((u128(w) << 64) / q); }

bool is_prime(uint64_t n) {
    if (n < 2) return false;
    static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t p : bases) {
        if (n == p) return true;
        if (n % p == 0) return false;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        ++s;
    }
    for (uint64_t a : bases) {
        uint64_t x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool composite = true;
        for (int i = 1; i < s; ++i) {
            x = mulmod(x, x, n);
            if (x == n - 1) {
                composite = false;
                break;
            }
        }
        if (composite) return false;
    }
    return true;
}

bool get_primes(uint32_t ntt_size, int bit_size, uint32_t count, std::vector<uint64_t>& out) {
    out.clear();
    if (bit_size < 2 || bit_size > 62) return false;
    const uint64_t step = 2ull * ntt_size;
    uint64_t v = (1ull << bit_size) - step + 1;
    const uint64_t lower = 1ull << (bit_size - 1);
    while (out.size() < count && v > lower) {
        if (is_prime(v)) out.push_back(v);
        v -= step;
    }
    return out.size() == count;
}

uint64_t minimal_primitive_root(uint64_t degree, uint64_t q) {
    if (degree == 0 || (q - 1) % degree) return 0;
    const uint64_t cof = (q - 1) / degree;
    uint64_t root = 0;
    for (uint64_t g = 2; g < q; ++g) {
        const uint64_t c = powmod(g, cof, q);
        if (powmod(c, degree >> 1, q) == q - 1) {
            root = c;
            break;
        }
    }
    if (!root) return 0;
    // the minimum over the odd powers of any primitive root is unique
    const uint64_t sq = mulmod(root, root, q);
    uint64_t cur = root, best = root;
    for (uint64_t i = 0; i < degree; ++i) {
        if (cur < best) best = cur;
        cur = mulmod(cur, sq, q);
    }
    return best;
}

uint32_t bit_reverse(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) {
        r = (r << 1) | (x & 1u);
        x >>= 1;
    }
    return r;
}

void barrett_ratio(uint64_t q, uint64_t& r0, uint64_t& r1) {
    // floor(2^128 / q) as two words
    const u128 hi = (~u128(0)) / q;  // floor((2^128 - 1) / q) == floor(2^128 / q) for q not a power of 2
    r0 = static_cast<uint64_t>(hi);
    r1 = static_cast<uint64_t>(hi >> 64);
}

bool make_ntt_tables(uint32_t n, uint64_t q, NttTables& t) {
    int logn = 0;
    while ((1u << logn) < n) ++logn;
    if ((1u << logn) != n) return false;
    const uint64_t root = minimal_primitive_root(2ull * n, q);
    if (!root) return false;
    const uint64_t iroot = invmod(root, q);
    t.n = n;
    t.q = q;
    t.root = root;
    t.rp.assign(n, 0);
    t.irp.assign(n, 0);
    t.rp_sh.assign(n, 0);
    t.irp_sh.assign(n, 0);
    uint64_t pw = root, ipw = iroot;
    t.rp[0] = 1;
    t.irp[0] = 1;
    for (uint32_t i = 1; i < n; ++i) {
        t.rp[bit_reverse(i, logn)] = pw;
        t.irp[bit_reverse(i, logn)] = ipw;
        pw = mulmod(pw, root, q);
        ipw = mulmod(ipw, iroot, q);
    }
    t.n_inv = invmod(n, q);
    t.n_inv_sh = shoup(t.n_inv, q);
    t.irp[1] = mulmod(t.irp[1], t.n_inv, q);
    for (uint32_t i = 0; i < n; ++i) {
        t.rp_sh[i] = shoup(t.rp[i], q);
        t.irp_sh[i] = shoup(t.irp[i], q);
    }
    barrett_ratio(q, t.ratio0, t.ratio1);
    return true;
}

void ntt_forward_host(uint64_t* a, const NttTables& t) {
    const uint32_t n = t.n;
    const uint64_t q = t.q;
    for (uint32_t m = 1; m < n; m <<= 1) {
        const uint32_t h = n / (2 * m);
        for (uint32_t k = 0; k < m; ++k) {
            const uint64_t w = t.rp[m + k];
            for (uint32_t j = 2 * k * h; j < 2 * k * h + h; ++j) {
                const uint64_t u = a[j], v = mulmod(a[j + h], w, q);
                a[j] = (u + v) % q;
                a[j + h] = (u + q - v) % q;
            }
        }
    }
}

void ntt_inverse_host(uint64_t* a, const NttTables& t) {
    const uint32_t n = t.n;
    const uint64_t q = t.q;
    for (uint32_t m = n / 2; m >= 1; m >>= 1) {
        const uint32_t h = n / (2 * m);
        for (uint32_t k = 0; k < m; ++k) {
            const uint64_t w = t.irp[m + k];
            for (uint32_t j = 2 * k * h; j < 2 * k * h + h; ++j) {
                const uint64_t u = a[j], v = a[j + h];
                a[j] = (u + v) % q;
                a[j + h] = mulmod((u + q - v) % q, w, q);
            }
        }
        if (m == 1) break;
    }
    for (uint32_t j = 0; j < n / 2; ++j) a[j] = mulmod(a[j], t.n_inv, q);
}

}  // namespace host
}  // namespace cbs
