/*
 * oracle.c -- CPU restatement of the reference's bootstrapping hot path.
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the CUDA path and the
 * timed CPU baseline; never linked into or called by the product library.
 *
 * Exact integer arithmetic throughout (unsigned __int128).  Batched routines use
 * OpenMP over independent ciphertexts.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------------------------ */
/* scalar modular arithmetic                                                                    */
/* ------------------------------------------------------------------------------------------ */

uint64_t orc_mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }

static inline uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    return (s >= q || s < a) ? s - q : s;
}
static inline uint64_t submod(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : a + q - b; }

uint64_t orc_powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = orc_mulmod(r, a, q);
        a = orc_mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}

uint64_t orc_invmod(uint64_t a, uint64_t q) {
    /* extended Euclid over signed 128-bit */
    __int128 t = 0, nt = 1, r = q, nr = a % q;
    while (nr != 0) {
        __int128 quo = r / nr, tmp;
        tmp = t - quo * nt; t = nt; nt = tmp;
        tmp = r - quo * nr; r = nr; nr = tmp;
    }
    if (r != 1) return 0;
    if (t < 0) t += q;
    return (uint64_t)t;
}

/* floor(w * 2^64 / q): the Shoup quotient (src/host/uintarithsmallmod.h compute_shoup) */
uint64_t orc_shoup(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

/* deterministic Miller-Rabin for 64-bit integers (bases valid for n < 2^64) */
int orc_is_prime(uint64_t n) {
    if (n < 2) return 0;
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (size_t i = 0; i < sizeof(small) / sizeof(small[0]); ++i) {
        if (n == small[i]) return 1;
        if (n % small[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; ++s; }
    for (size_t i = 0; i < sizeof(small) / sizeof(small[0]); ++i) {
        uint64_t x = orc_powmod(small[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int r = 1; r < s; ++r) {
            x = orc_mulmod(x, x, n);
            if (x == n - 1) { comp = 0; break; }
        }
        if (comp) return 0;
    }
    return 1;
}

/* src/host/numth.cu:207-233: start at 2^bits - 2N + 1 and step down by 2N */
int orc_get_primes(uint32_t ntt_size, int bit_size, uint32_t count, uint64_t *out) {
    const uint64_t factor = 2ull * ntt_size;
    uint64_t value = (1ull << bit_size) - factor + 1;
    const uint64_t lower = 1ull << (bit_size - 1);
    uint32_t found = 0;
    while (found < count && value > lower) {
        if (orc_is_prime(value)) out[found++] = value;
        value -= factor;
    }
    return found == count ? 0 : -1;
}

/* src/host/numth.cu:309-331: the smallest primitive degree-th root of unity. The reference
 * starts from a random primitive root and scans its odd powers; the minimum over that orbit
 * does not depend on the starting root, so a deterministic search gives the same value. */
uint64_t orc_minimal_primitive_root(uint64_t degree, uint64_t q) {
    if ((q - 1) % degree) return 0;
    const uint64_t cof = (q - 1) / degree;
    uint64_t root = 0;
    for (uint64_t g = 2; g < q; ++g) {
        uint64_t c = orc_powmod(g, cof, q);
        if (orc_powmod(c, degree >> 1, q) == q - 1) { root = c; break; }
    }
    if (!root) return 0;
    const uint64_t gsq = orc_mulmod(root, root, q);
    uint64_t cur = root, best = root;
    for (uint64_t i = 0; i < degree; ++i) {
        if (cur < best) best = cur;
        cur = orc_mulmod(cur, gsq, q);
    }
    return best;
}

/* ------------------------------------------------------------------------------------------ */
/* Phantom NTT tables and transforms                                                           */
/* ------------------------------------------------------------------------------------------ */

static inline uint32_t brev(uint32_t x, uint32_t bits) {
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* src/host/ntt.cu:11-56 */
int orc_ntt_tables(uint32_t log_n, uint64_t q, uint64_t *rp, uint64_t *rp_sh, uint64_t *irp, uint64_t *irp_sh,
                   uint64_t *n_inv) {
    const uint32_t n = 1u << log_n;
    const uint64_t root = orc_minimal_primitive_root(2ull * n, q);
    if (!root) return -1;
    const uint64_t iroot = orc_invmod(root, q);
    uint64_t pw = root, ipw = iroot;
    rp[0] = 1;
    irp[0] = 1;
    for (uint32_t i = 1; i < n; ++i) {
        rp[brev(i, log_n)] = pw;
        irp[brev(i, log_n)] = ipw;
        pw = orc_mulmod(pw, root, q);
        ipw = orc_mulmod(ipw, iroot, q);
    }
    const uint64_t ninv = orc_invmod(n, q);
    irp[1] = orc_mulmod(irp[1], ninv, q);
    for (uint32_t i = 0; i < n; ++i) {
        if (rp_sh) rp_sh[i] = orc_shoup(rp[i], q);
        if (irp_sh) irp_sh[i] = orc_shoup(irp[i], q);
    }
    n_inv[0] = ninv;
    n_inv[1] = orc_shoup(ninv, q);
    return 0;
}

/* ntt_1d.cu:488-555: Cooley-Tukey, twiddle rp[m+k] for group k of stage m */
static void ntt_fwd_one(uint64_t *a, uint32_t n, uint64_t q, const uint64_t *rp) {
    for (uint32_t m = 1; m < n; m <<= 1) {
        const uint32_t t = n / (2 * m);
        for (uint32_t k = 0; k < m; ++k) {
            const uint64_t w = rp[m + k];
            for (uint32_t j = 2 * k * t; j < 2 * k * t + t; ++j) {
                const uint64_t u = a[j], v = orc_mulmod(a[j + t], w, q);
                a[j] = addmod(u, v, q);
                a[j + t] = submod(u, v, q);
            }
        }
    }
}

/* ntt_1d.cu:557-617: Gentleman-Sande; the last stage scales x by n^-1 and y through irp[1] */
static void ntt_inv_one(uint64_t *a, uint32_t n, uint64_t q, const uint64_t *irp, uint64_t n_inv) {
    for (uint32_t m = n / 2; m >= 1; m >>= 1) {
        const uint32_t t = n / (2 * m);
        for (uint32_t k = 0; k < m; ++k) {
            const uint64_t w = irp[m + k];
            for (uint32_t j = 2 * k * t; j < 2 * k * t + t; ++j) {
                const uint64_t u = a[j], v = a[j + t];
                a[j] = addmod(u, v, q);
                a[j + t] = orc_mulmod(submod(u, v, q), w, q);
            }
        }
        if (m == 1) break;
    }
    for (uint32_t j = 0; j < n / 2; ++j) a[j] = orc_mulmod(a[j], n_inv, q);
}

void orc_ntt_forward(uint64_t *a, size_t batch, uint32_t n, uint64_t q, const uint64_t *rp) {
#pragma omp parallel for schedule(static)
    for (long b = 0; b < (long)batch; ++b) ntt_fwd_one(a + (size_t)b * n, n, q, rp);
}

void orc_ntt_inverse(uint64_t *a, size_t batch, uint32_t n, uint64_t q, const uint64_t *irp, uint64_t n_inv) {
#pragma omp parallel for schedule(static)
    for (long b = 0; b < (long)batch; ++b) ntt_inv_one(a + (size_t)b * n, n, q, irp, n_inv);
}

void orc_ntt_inverse_permute(uint64_t *out, const uint64_t *in, const uint32_t *map, size_t batch, uint32_t n,
                             uint64_t q, const uint64_t *irp, uint64_t n_inv) {
#pragma omp parallel for schedule(static)
    for (long b = 0; b < (long)batch; ++b) {
        const uint64_t *src = in + (size_t)b * n;
        uint64_t *dst = out + (size_t)b * n;
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t s = map[i];
            int neg = 0;
            if (s >= n) { s -= n; neg = 1; }
            uint64_t v = src[s];
            dst[i] = (neg && v) ? q - v : v;
        }
        ntt_inv_one(dst, n, q, irp, n_inv);
    }
}

void orc_negacyclic_mul(const uint64_t *a, const uint64_t *b, uint64_t *c, uint32_t n, uint64_t q) {
    u128 *acc = (u128 *)calloc(2 * (size_t)n, sizeof(u128));
    /* accumulate positive and negative halves separately, reduce at the end */
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t j = 0; j < n; ++j) {
            const u128 p = (u128)a[i] * b[j];
            const uint32_t k = i + j;
            if (k < n) acc[k] += p % q;
            else acc[n + (k - n)] += p % q;
        }
    }
    for (uint32_t k = 0; k < n; ++k) c[k] = submod((uint64_t)(acc[k] % q), (uint64_t)(acc[n + k] % q), q);
    free(acc);
}

/* kernel.cu:7554-7571 */
void orc_auto_maps(uint32_t *maps, uint32_t n, uint32_t levels) {
    uint32_t log_n = 0;
    while ((1u << log_n) < n) ++log_n;
    for (uint32_t lv = 0; lv < levels; ++lv) {
        const uint64_t k = (uint64_t)(n >> lv) + 1;
        for (uint32_t tid = 0; tid < n; ++tid) {
            const uint32_t j = brev(tid, log_n);
            const uint64_t jt = 2ull * j + 1;
            const uint32_t idx = (uint32_t)(((jt * k) & (2ull * n - 1)) >> 1);
            maps[(size_t)lv * n + tid] = brev(idx, log_n);
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* gadget decomposition and modulus switching                                                  */
/* ------------------------------------------------------------------------------------------ */

/* kernel.cu:37-68 (and the identical device_SignedDigitDecompose, kernel.cu:768-798) */
void orc_signed_decompose(uint64_t x, uint64_t Q, uint32_t base, uint32_t digits, uint64_t *out) {
    const int gbits = __builtin_ctz(base);
    const int logq = 64 - __builtin_clzll(Q);
    int ign = logq - (int)digits * gbits;
    if (ign < 0) ign = 0;
    const uint64_t qhalf = Q >> 1;
    const int64_t qi = (int64_t)Q;
    int64_t d = x < qhalf ? (int64_t)x : (int64_t)x - qi;
    int64_t r;
    if (ign != 0) {
        r = (int64_t)((uint64_t)d << (64 - ign)) >> (64 - ign);
        d = (d - r) >> ign;
    }
    for (uint32_t i = 0; i < digits; ++i) {
        r = (int64_t)((uint64_t)d << (64 - gbits)) >> (64 - gbits);
        d = (d - r) >> gbits;
        if (r < 0) r += qi;
        out[i] = (uint64_t)r;
    }
}

/* kernel.cu:7316-7326 */
uint32_t orc_special_ms(uint64_t v, uint32_t two_n, uint64_t q, uint32_t bitwidth) {
    const uint64_t shift = bitwidth < 63u ? (1ull << bitwidth) : 0ull;
    if (shift == 0 || two_n == 0 || q == 0) return 0;
    const double scale = (double)two_n / ((double)q * (double)shift);
    const double x = (double)v * scale;
    const uint64_t r = (uint64_t)floor(x + 0.5);
    return (uint32_t)((r * shift) & ((uint64_t)two_n - 1));
}

/* ------------------------------------------------------------------------------------------ */
/* circuit bootstrapping                                                                       */
/* ------------------------------------------------------------------------------------------ */

/* NTT of the monic polynomial X^e - 1 (e in [0, 2N)), OpenFHE convention (cirbts-init.cu:991-1023) */
static void monic_ntt(uint64_t *out, uint32_t e, uint32_t N, uint64_t Q, const uint64_t *rp) {
    memset(out, 0, sizeof(uint64_t) * N);
    if (e < N) out[e] = addmod(out[e], 1, Q);
    else out[e - N] = submod(out[e - N], 1, Q);
    out[0] = submod(out[0], 1, Q);
    ntt_fwd_one(out, N, Q, rp);
}

/* X^{-e} * p in the coefficient domain (negacyclic rotation), e in [0, 2N) */
static void rotate_neg(uint64_t *out, const uint64_t *p, uint32_t e, uint32_t N, uint64_t Q) {
    for (uint32_t i = 0; i < N; ++i) {
        /* out[i] = coefficient of X^i in X^{-e} p = p[i+e] with sign */
        uint32_t s = (i + e) % (2 * N);
        uint64_t v = s < N ? p[s] : p[s - N];
        out[i] = (s < N) ? v : (v ? Q - v : 0);
    }
}

static void blind_rotate_one(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *a, uint64_t b,
                             uint64_t *acc, int finalize, uint64_t *work) {
    const uint32_t N = p->N, l2 = 2 * p->digits_g;
    const uint64_t Q = p->Q;
    const uint32_t twoN = 2 * N;
    const uint32_t bw = (p->num_lut <= 1) ? 0 : (uint32_t)(32 - __builtin_clz(p->num_lut - 1));
    uint64_t *ct = work;              /* [2][N] */
    uint64_t *dct = ct + 2 * N;       /* [l2][N] */
    uint64_t *mono = dct + (size_t)l2 * N;
    uint64_t dig[64];

    /* acc = (0, LUT * X^{-b~}) : kernel.cu:7328-7358 */
    const uint32_t bt = orc_special_ms(b, twoN, p->q_lwe, bw);
    memset(acc, 0, sizeof(uint64_t) * N);
    rotate_neg(acc + N, k->tv, bt, N, Q);
    ntt_fwd_one(acc + N, N, Q, k->rp);

    for (uint32_t i = 0; i < p->n; ++i) {
        /* INTT(acc) -> signed digits -> NTT (kernel.cu:473-559) */
        memcpy(ct, acc, sizeof(uint64_t) * 2 * N);
        ntt_inv_one(ct, N, Q, k->irp, k->n_inv);
        ntt_inv_one(ct + N, N, Q, k->irp, k->n_inv);
        for (uint32_t poly = 0; poly < 2; ++poly) {
            for (uint32_t c = 0; c < N; ++c) {
                orc_signed_decompose(ct[poly * N + c], Q, p->base_g, p->digits_g, dig);
                for (uint32_t j = 0; j < p->digits_g; ++j) dct[(size_t)(2 * j + poly) * N + c] = dig[j];
            }
        }
        for (uint32_t d = 0; d < l2; ++d) ntt_fwd_one(dct + (size_t)d * N, N, Q, k->rp);
        /* MAC against BSK_i, times (X^{a~_i} - 1), accumulate (kernel.cu:3008-3055) */
        const uint32_t at = orc_special_ms(a[i], twoN, p->q_lwe, bw);
        monic_ntt(mono, at, N, Q, k->rp);
        const uint64_t *ek = k->bsk + (size_t)i * l2 * 2 * N;
        for (uint32_t c = 0; c < N; ++c) {
            uint64_t t0 = 0, t1 = 0;
            for (uint32_t d = 0; d < l2; ++d) {
                const uint64_t x = dct[(size_t)d * N + c];
                t0 = addmod(t0, orc_mulmod(x, ek[(size_t)d * 2 * N + c], Q), Q);
                t1 = addmod(t1, orc_mulmod(x, ek[(size_t)d * 2 * N + N + c], Q), Q);
            }
            acc[c] = addmod(acc[c], orc_mulmod(t0, mono[c], Q), Q);
            acc[N + c] = addmod(acc[N + c], orc_mulmod(t1, mono[c], Q), Q);
        }
    }

    if (finalize) {
        /* cirbts-batch.cu:2622-2642: x N^-1, INTT, c1[i] += (gpow[i]>>1) N^-1, NTT */
        const uint64_t ninv = orc_invmod(N, Q);
        for (uint32_t c = 0; c < 2 * N; ++c) acc[c] = orc_mulmod(acc[c], ninv, Q);
        ntt_inv_one(acc, N, Q, k->irp, k->n_inv);
        ntt_inv_one(acc + N, N, Q, k->irp, k->n_inv);
        for (uint32_t j = 0; j < p->num_lut; ++j)
            acc[N + j] = addmod(acc[N + j], orc_mulmod(k->gpow[j] >> 1, ninv, Q), Q);
        ntt_fwd_one(acc, N, Q, k->rp);
        ntt_fwd_one(acc + N, N, Q, k->rp);
    }
}

void orc_blind_rotate(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *a, const uint64_t *b,
                      uint32_t batch, uint32_t a_stride, uint64_t *acc_out, int finalize) {
    const size_t wsz = (size_t)(2 + 2 * p->digits_g + 1) * p->N;
#pragma omp parallel
    {
        uint64_t *work = (uint64_t *)malloc(wsz * sizeof(uint64_t));
#pragma omp for schedule(dynamic, 1)
        for (long bi = 0; bi < (long)batch; ++bi)
            blind_rotate_one(p, k, a + (size_t)bi * a_stride, b[bi], acc_out + (size_t)bi * 2 * p->N, finalize, work);
        free(work);
    }
}

/* Multi-bit blind rotation (the reference's CIRBTS_PBS_MULTIBIT = 2 / 3 / 4 path: key grouping
 * cirbts-init.cu:376-565, MB3 MAC kernel.cu:4585-4771, MB4 staging cirbts-batch.cu:2767-2923).
 * For binary s_i, prod_{i in G} (1 + (X^{a_i} - 1) s_i) = X^{sum a_i s_i}, so one step per
 * group G of mb coefficients adds sum_S m_S (acc (x) RGSW(prod_{i in S} s_i)) with m_S =
 * prod_{i in S} (X^{a_i} - 1) over the non-empty subsets S, in the order {0} {1} {2} {0,1}
 * {0,2} {1,2} {0,1,2} (mb = 3) or {0} {1} {0,1} (mb = 2).  mb = 4 is the reference's staged
 * grouping: 8 keys per group of 4, {0} {1} {2} {3} {0,1} {0,2} {1,2} {0,1,2}; the group adds
 * the mb = 3 step of coefficients 0-2 (keys 0 1 2 4 5 6 7), then a one-bit step of
 * coefficient 3 (key 3) on a fresh decomposition of the updated accumulator.  Coefficients
 * past n rotate by 0, so their subsets vanish.  mbk [groups][keys][2*digits_g][2][N] NTT domain. */
static const uint32_t orc_mb_order2[3] = {1u, 2u, 3u};
static const uint32_t orc_mb_order3[7] = {1u, 2u, 4u, 3u, 5u, 6u, 7u};
static const uint32_t orc_mb_order4[8] = {1u, 2u, 4u, 8u, 3u, 5u, 6u, 7u};

uint32_t orc_mb_keys(uint32_t mb) { return mb == 4 ? 8u : (1u << mb) - 1u; }

uint32_t orc_mb_mask(uint32_t mb, uint32_t kk) {
    return mb == 2 ? orc_mb_order2[kk] : (mb == 3 ? orc_mb_order3[kk] : (mb == 4 ? orc_mb_order4[kk] : 1u));
}

/* one step: decompose acc, then acc += sum over the step's keys of m_mask (acc (x) key), the
 * monomials of the nc coefficients idx0 .. idx0 + nc - 1 */
static void mb_step(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *a, uint32_t idx0, uint32_t nc,
                    const uint64_t *gk, const uint32_t *slots, const uint32_t *masks, uint32_t nkeys, uint64_t *acc,
                    uint64_t *work) {
    const uint32_t N = p->N, l2 = 2 * p->digits_g, twoN = 2 * N;
    const uint64_t Q = p->Q;
    const uint32_t bw = (p->num_lut <= 1) ? 0 : (uint32_t)(32 - __builtin_clz(p->num_lut - 1));
    uint64_t *ct = work;                    /* [2][N] */
    uint64_t *dct = ct + 2 * N;             /* [l2][N] */
    uint64_t *mono = dct + (size_t)l2 * N;  /* [nc][N] */
    uint64_t *msub = mono + (size_t)3 * N;  /* [nkeys][N] */
    uint64_t dig[64];
    memcpy(ct, acc, sizeof(uint64_t) * 2 * N);
    ntt_inv_one(ct, N, Q, k->irp, k->n_inv);
    ntt_inv_one(ct + N, N, Q, k->irp, k->n_inv);
    for (uint32_t poly = 0; poly < 2; ++poly)
        for (uint32_t c = 0; c < N; ++c) {
            orc_signed_decompose(ct[poly * N + c], Q, p->base_g, p->digits_g, dig);
            for (uint32_t j = 0; j < p->digits_g; ++j) dct[(size_t)(2 * j + poly) * N + c] = dig[j];
        }
    for (uint32_t d = 0; d < l2; ++d) ntt_fwd_one(dct + (size_t)d * N, N, Q, k->rp);
    for (uint32_t i = 0; i < nc; ++i) {
        const uint32_t idx = idx0 + i;
        const uint32_t at = idx < p->n ? orc_special_ms(a[idx], twoN, p->q_lwe, bw) : 0u;
        monic_ntt(mono + (size_t)i * N, at, N, Q, k->rp);
    }
    for (uint32_t kk = 0; kk < nkeys; ++kk) {
        uint64_t *m = msub + (size_t)kk * N;
        for (uint32_t c = 0; c < N; ++c) m[c] = 1;
        for (uint32_t i = 0; i < nc; ++i)
            if (masks[kk] & (1u << i))
                for (uint32_t c = 0; c < N; ++c) m[c] = orc_mulmod(m[c], mono[(size_t)i * N + c], Q);
    }
    for (uint32_t c = 0; c < N; ++c) {
        uint64_t u0 = 0, u1 = 0;
        for (uint32_t kk = 0; kk < nkeys; ++kk) {
            const uint64_t *ek = gk + (size_t)slots[kk] * l2 * 2 * N;
            uint64_t t0 = 0, t1 = 0;
            for (uint32_t d = 0; d < l2; ++d) {
                const uint64_t x = dct[(size_t)d * N + c];
                t0 = addmod(t0, orc_mulmod(x, ek[(size_t)d * 2 * N + c], Q), Q);
                t1 = addmod(t1, orc_mulmod(x, ek[(size_t)d * 2 * N + N + c], Q), Q);
            }
            u0 = addmod(u0, orc_mulmod(t0, msub[(size_t)kk * N + c], Q), Q);
            u1 = addmod(u1, orc_mulmod(t1, msub[(size_t)kk * N + c], Q), Q);
        }
        acc[c] = addmod(acc[c], u0, Q);
        acc[N + c] = addmod(acc[N + c], u1, Q);
    }
}

static void blind_rotate_mb_one(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *mbk, uint32_t mb,
                                const uint64_t *a, uint64_t b, uint64_t *acc, int finalize, uint64_t *work) {
    static const uint32_t id_slots[7] = {0u, 1u, 2u, 3u, 4u, 5u, 6u};
    static const uint32_t mb4_slots_a[7] = {0u, 1u, 2u, 4u, 5u, 6u, 7u};
    static const uint32_t mb4_slot_b[1] = {3u}, one_mask[1] = {1u};
    const uint32_t N = p->N, l2 = 2 * p->digits_g, K = orc_mb_keys(mb);
    const uint32_t groups = (p->n + mb - 1) / mb;
    const uint64_t Q = p->Q;
    const uint32_t twoN = 2 * N;
    const uint32_t bw = (p->num_lut <= 1) ? 0 : (uint32_t)(32 - __builtin_clz(p->num_lut - 1));

    const uint32_t bt = orc_special_ms(b, twoN, p->q_lwe, bw);
    memset(acc, 0, sizeof(uint64_t) * N);
    rotate_neg(acc + N, k->tv, bt, N, Q);
    ntt_fwd_one(acc + N, N, Q, k->rp);

    for (uint32_t g = 0; g < groups; ++g) {
        const uint64_t *gk = mbk + (size_t)g * K * l2 * 2 * N;
        if (mb == 4) {
            mb_step(p, k, a, 4 * g, 3, gk, mb4_slots_a, orc_mb_order3, 7, acc, work);
            if (4 * g + 3 < p->n) mb_step(p, k, a, 4 * g + 3, 1, gk, mb4_slot_b, one_mask, 1, acc, work);
        } else {
            mb_step(p, k, a, g * mb, mb, gk, id_slots, mb == 2 ? orc_mb_order2 : orc_mb_order3, K, acc, work);
        }
    }

    if (finalize) {
        const uint64_t ninv = orc_invmod(N, Q);
        for (uint32_t c = 0; c < 2 * N; ++c) acc[c] = orc_mulmod(acc[c], ninv, Q);
        ntt_inv_one(acc, N, Q, k->irp, k->n_inv);
        ntt_inv_one(acc + N, N, Q, k->irp, k->n_inv);
        for (uint32_t j = 0; j < p->num_lut; ++j)
            acc[N + j] = addmod(acc[N + j], orc_mulmod(k->gpow[j] >> 1, ninv, Q), Q);
        ntt_fwd_one(acc, N, Q, k->rp);
        ntt_fwd_one(acc + N, N, Q, k->rp);
    }
}

void orc_blind_rotate_mb(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *mbk, uint32_t mb,
                         const uint64_t *a, const uint64_t *b, uint32_t batch, uint32_t a_stride, uint64_t *acc_out,
                         int finalize) {
    const size_t wsz = (size_t)(2 + 2 * p->digits_g + 3 + orc_mb_keys(mb)) * p->N;
#pragma omp parallel
    {
        uint64_t *work = (uint64_t *)malloc(wsz * sizeof(uint64_t));
#pragma omp for schedule(dynamic, 1)
        for (long bi = 0; bi < (long)batch; ++bi)
            blind_rotate_mb_one(p, k, mbk, mb, a + (size_t)bi * a_stride, b[bi], acc_out + (size_t)bi * 2 * p->N,
                                finalize, work);
        free(work);
    }
}

/* one HomTrace + SchemeSwitch pipeline for a single MV RLWE (cirbts-batch.cu:1656-1789,
 * kernel.cu:7832-7888 HT update, kernel.cu:8407-8446 SS update, kernel.cu:7776-7789 layout) */
static void trace_ss_one(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *ct_in, uint64_t *rgsw,
                         uint64_t *work) {
    const uint32_t N = p->N;
    const uint64_t Q = p->Q;
    uint64_t *c0 = work, *c1 = c0 + N, *perm = c1 + N, *pc1 = perm + N;
    const uint32_t maxd = p->digits_ht > p->digits_ss ? p->digits_ht : p->digits_ss;
    uint64_t *dg = pc1 + N; /* [maxd][N] */
    uint64_t dig[64];
    memcpy(c0, ct_in, sizeof(uint64_t) * N);
    memcpy(c1, ct_in + N, sizeof(uint64_t) * N);

    for (uint32_t r = 0; r < p->trace_rounds; ++r) {
        const uint32_t *map = k->auto_maps + (size_t)r * N;
        /* sigma(c0) in the coefficient domain */
        for (uint32_t i = 0; i < N; ++i) perm[i] = c0[map[i]];
        ntt_inv_one(perm, N, Q, k->irp, k->n_inv);
        for (uint32_t c = 0; c < N; ++c) {
            orc_signed_decompose(perm[c], Q, p->base_ht, p->digits_ht, dig);
            for (uint32_t j = 0; j < p->digits_ht; ++j) dg[(size_t)j * N + c] = dig[j];
        }
        for (uint32_t j = 0; j < p->digits_ht; ++j) ntt_fwd_one(dg + (size_t)j * N, N, Q, k->rp);
        const uint64_t *key = k->ht_key + (size_t)r * p->digits_ht * 2 * N;
        for (uint32_t i = 0; i < N; ++i) pc1[i] = c1[map[i]];
        for (uint32_t c = 0; c < N; ++c) {
            uint64_t s0 = 0, s1 = 0;
            for (uint32_t j = 0; j < p->digits_ht; ++j) {
                const uint64_t x = dg[(size_t)j * N + c];
                s0 = addmod(s0, orc_mulmod(x, key[(size_t)j * 2 * N + c], Q), Q);
                s1 = addmod(s1, orc_mulmod(x, key[(size_t)j * 2 * N + N + c], Q), Q);
            }
            c0[c] = addmod(c0[c], s0, Q);
            c1[c] = addmod(addmod(c1[c], s1, Q), pc1[c], Q);
        }
    }
    /* trace result -> RGSW row 2j+1 */
    memcpy(rgsw + 2 * N, c0, sizeof(uint64_t) * N);
    memcpy(rgsw + 3 * N, c1, sizeof(uint64_t) * N);

    /* SchemeSwitch: digits(INTT(c0)) x SSkey; row 2j = (c1 + ks0, ks1) */
    memcpy(perm, c0, sizeof(uint64_t) * N);
    ntt_inv_one(perm, N, Q, k->irp, k->n_inv);
    for (uint32_t c = 0; c < N; ++c) {
        orc_signed_decompose(perm[c], Q, p->base_ss, p->digits_ss, dig);
        for (uint32_t j = 0; j < p->digits_ss; ++j) dg[(size_t)j * N + c] = dig[j];
    }
    for (uint32_t j = 0; j < p->digits_ss; ++j) ntt_fwd_one(dg + (size_t)j * N, N, Q, k->rp);
    for (uint32_t c = 0; c < N; ++c) {
        uint64_t s0 = 0, s1 = 0;
        for (uint32_t j = 0; j < p->digits_ss; ++j) {
            const uint64_t x = dg[(size_t)j * N + c];
            s0 = addmod(s0, orc_mulmod(x, k->ss_key[(size_t)j * 2 * N + c], Q), Q);
            s1 = addmod(s1, orc_mulmod(x, k->ss_key[(size_t)j * 2 * N + N + c], Q), Q);
        }
        rgsw[c] = addmod(c1[c], s0, Q);
        rgsw[N + c] = s1;
    }
    (void)maxd;
}

static size_t trace_work_words(const orc_cbs_params *p) {
    const uint32_t maxd = p->digits_ht > p->digits_ss ? p->digits_ht : p->digits_ss;
    return (size_t)(4 + maxd) * p->N;
}

void orc_trace_schemeswitch(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *ct, uint32_t count,
                            uint64_t *rgsw_out) {
    const size_t wsz = trace_work_words(p);
#pragma omp parallel
    {
        uint64_t *work = (uint64_t *)malloc(wsz * sizeof(uint64_t));
#pragma omp for schedule(dynamic, 1)
        for (long i = 0; i < (long)count; ++i)
            trace_ss_one(p, k, ct + (size_t)i * 2 * p->N, rgsw_out + (size_t)i * 4 * p->N, work);
        free(work);
    }
}

/* BR + finalize + MV split: kernel.cu:7498-7536 ct_j = acc * X^{-j} (NTT domain) */
void orc_blind_rotate_mv(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *a, const uint64_t *b,
                         uint32_t batch, uint32_t a_stride, uint64_t *mv) {
    const uint32_t N = p->N, L = p->num_lut;
    const uint64_t Q = p->Q;
    uint64_t *acc = (uint64_t *)malloc(sizeof(uint64_t) * 2 * N * batch);
    orc_blind_rotate(p, k, a, b, batch, a_stride, acc, 1);
    uint64_t *mono = (uint64_t *)malloc(sizeof(uint64_t) * N * L);
    for (uint32_t j = 0; j < L; ++j) {
        uint64_t *m = mono + (size_t)j * N;
        memset(m, 0, sizeof(uint64_t) * N);
        if (j == 0) m[0] = 1;
        else m[N - j] = Q - 1; /* X^{-j} = -X^{N-j} */
        ntt_fwd_one(m, N, Q, k->rp);
    }
    for (uint32_t bi = 0; bi < batch; ++bi)
        for (uint32_t j = 0; j < L; ++j)
            for (uint32_t poly = 0; poly < 2; ++poly)
                for (uint32_t c = 0; c < N; ++c)
                    mv[(((size_t)bi * L + j) * 2 + poly) * N + c] =
                        orc_mulmod(acc[((size_t)bi * 2 + poly) * N + c], mono[(size_t)j * N + c], Q);
    free(mono);
    free(acc);
}

void orc_circuit_bootstrap(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *a, const uint64_t *b,
                           uint32_t batch, uint32_t a_stride, uint64_t *rgsw_out) {
    uint64_t *mv = (uint64_t *)malloc(sizeof(uint64_t) * 2 * p->N * (size_t)batch * p->num_lut);
    orc_blind_rotate_mv(p, k, a, b, batch, a_stride, mv);
    orc_trace_schemeswitch(p, k, mv, batch * p->num_lut, rgsw_out);
    free(mv);
}

/* ------------------------------------------------------------------------------------------ */
/* CMux LUT                                                                                    */
/* ------------------------------------------------------------------------------------------ */

void orc_external_product(const uint64_t *ct_in, const uint64_t *rgsw, uint64_t *out, uint32_t N, uint64_t Q,
                          const uint64_t *rp, const uint64_t *irp, uint64_t n_inv, uint32_t base, uint32_t digits) {
    uint64_t *ct = (uint64_t *)malloc(sizeof(uint64_t) * 2 * N);
    uint64_t *dct = (uint64_t *)malloc(sizeof(uint64_t) * 2 * digits * N);
    uint64_t dig[64];
    memcpy(ct, ct_in, sizeof(uint64_t) * 2 * N);
    ntt_inv_one(ct, N, Q, irp, n_inv);
    ntt_inv_one(ct + N, N, Q, irp, n_inv);
    for (uint32_t poly = 0; poly < 2; ++poly)
        for (uint32_t c = 0; c < N; ++c) {
            orc_signed_decompose(ct[poly * N + c], Q, base, digits, dig);
            for (uint32_t j = 0; j < digits; ++j) dct[(size_t)(2 * j + poly) * N + c] = dig[j];
        }
    for (uint32_t d = 0; d < 2 * digits; ++d) ntt_fwd_one(dct + (size_t)d * N, N, Q, rp);
    for (uint32_t c = 0; c < N; ++c) {
        uint64_t s0 = 0, s1 = 0;
        for (uint32_t r = 0; r < 2 * digits; ++r) {
            const uint64_t x = dct[(size_t)r * N + c];
            s0 = addmod(s0, orc_mulmod(x, rgsw[((size_t)r * 2 + 0) * N + c], Q), Q);
            s1 = addmod(s1, orc_mulmod(x, rgsw[((size_t)r * 2 + 1) * N + c], Q), Q);
        }
        out[c] = s0;
        out[N + c] = s1;
    }
    free(dct);
    free(ct);
}

void orc_lut8x32(const uint64_t *table, const uint64_t *const *ctrl, uint64_t *out, uint32_t N, uint64_t Q,
                 const uint64_t *rp, const uint64_t *irp, uint64_t n_inv, uint32_t base, uint32_t digits) {
    const size_t ctsz = 2 * (size_t)N;
    uint64_t *cur = (uint64_t *)malloc(sizeof(uint64_t) * 256 * ctsz);
    uint64_t *delta = (uint64_t *)malloc(sizeof(uint64_t) * ctsz);
    uint64_t *prod = (uint64_t *)malloc(sizeof(uint64_t) * ctsz);
    memcpy(cur, table, sizeof(uint64_t) * 256 * ctsz);
    uint32_t count = 256;
    for (uint32_t bit = 0; bit < 8; ++bit) {
        for (uint32_t i = 0; i < count / 2; ++i) {
            const uint64_t *c0 = cur + (size_t)(2 * i) * ctsz, *c1 = c0 + ctsz;
            for (size_t c = 0; c < ctsz; ++c) delta[c] = submod(c1[c], c0[c], Q);
            orc_external_product(delta, ctrl[bit], prod, N, Q, rp, irp, n_inv, base, digits);
            uint64_t *dst = cur + (size_t)i * ctsz;
            for (size_t c = 0; c < ctsz; ++c) dst[c] = addmod(c0[c], prod[c], Q);
        }
        count /= 2;
    }
    memcpy(out, cur, sizeof(uint64_t) * ctsz);
    free(prod);
    free(delta);
    free(cur);
}

/* ------------------------------------------------------------------------------------------ */
/* sample extract + key switch                                                                 */
/* ------------------------------------------------------------------------------------------ */

/* aes_gpu_ks.cuh:388-394 modswitch_u64_to_pow2_u16 */
static inline uint32_t ms_pow2(uint64_t v, double q_over_Q, uint32_t mask) {
    const double x = (double)v * q_over_Q;
    return ((uint32_t)nearbyint(x)) & mask;
}

void orc_extract_keyswitch(const uint64_t *words_coef, const uint32_t *info, uint32_t T, uint32_t N, uint64_t Q,
                           const uint16_t *ksk, uint32_t n, uint32_t base_ks_log2, uint32_t qks, uint64_t q_lwe,
                           uint64_t *out_a, uint64_t *out_b, uint32_t out_stride) {
    const double q_over_Q = (double)qks / (double)Q;
    const uint32_t mask = qks - 1, bmask = (1u << base_ks_log2) - 1;
    const uint32_t outlen = n + 1, base = 1u << base_ks_log2;
    const size_t stride_i = (size_t)base * outlen, stride_j = (size_t)N * stride_i;
    const int divisible = (q_lwe % qks) == 0;
    const uint64_t scale = divisible ? q_lwe / qks : 0;
#pragma omp parallel for schedule(dynamic, 4)
    for (long t = 0; t < (long)T; ++t) {
        const uint32_t word = info[t] >> 16, idx = info[t] & 0xFFFFu;
        const uint64_t *a = words_coef + (size_t)word * 2 * N, *bw = a + N;
        uint32_t *acc = (uint32_t *)calloc(outlen, sizeof(uint32_t));
        acc[n] = ms_pow2(bw[idx], q_over_Q, mask);
        for (uint32_t j = 0; j < N; ++j) {
            uint64_t v;
            if (j <= idx) v = a[idx - j];
            else { const uint64_t ak = a[N + idx - j]; v = ak ? Q - ak : 0; }
            const uint32_t ai = ms_pow2(v, q_over_Q, mask);
            const uint32_t d0 = ai & bmask, d1 = (ai >> base_ks_log2) & bmask;
            const uint16_t *k0 = ksk + (size_t)j * stride_i + (size_t)d0 * outlen;
            const uint16_t *k1 = ksk + stride_j + (size_t)j * stride_i + (size_t)d1 * outlen;
            for (uint32_t k = 0; k < outlen; ++k) acc[k] -= (uint32_t)k0[k] + (uint32_t)k1[k];
        }
        for (uint32_t k = 0; k < outlen; ++k) {
            const uint64_t v = acc[k] & mask;
            /* aes_gpu_ks.cuh:431-440 ks_u16_to_lwe (round-half-up division for non-divisible q) */
            const uint64_t val = divisible ? v * scale : (uint64_t)(((u128)v * q_lwe + (qks >> 1)) / qks);
            if (k == n) out_b[t] = val;
            else out_a[(size_t)t * out_stride + k] = val;
        }
        free(acc);
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Phantom RNS NTT and hybrid key switching                                                    */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    uint64_t *rp, *irp;
    uint64_t ninv;
} orc_tab;

static void tab_make(orc_tab *t, uint32_t log_n, uint64_t q) {
    const uint32_t n = 1u << log_n;
    t->rp = (uint64_t *)malloc(sizeof(uint64_t) * n);
    t->irp = (uint64_t *)malloc(sizeof(uint64_t) * n);
    uint64_t ni[2];
    orc_ntt_tables(log_n, q, t->rp, NULL, t->irp, NULL, ni);
    t->ninv = ni[0];
}

static void tab_free(orc_tab *t) {
    free(t->rp);
    free(t->irp);
}

void orc_rns_ntt(uint64_t *data, size_t polys, uint32_t limbs, uint32_t log_n, const uint64_t *q, int inverse) {
    const uint32_t n = 1u << log_n;
    orc_tab *tabs = (orc_tab *)malloc(sizeof(orc_tab) * limbs);
    for (uint32_t l = 0; l < limbs; ++l) tab_make(&tabs[l], log_n, q[l]);
#pragma omp parallel for schedule(dynamic, 1)
    for (long i = 0; i < (long)(polys * limbs); ++i) {
        const uint32_t l = (uint32_t)(i % limbs);
        uint64_t *a = data + (size_t)i * n;
        if (inverse) ntt_inv_one(a, n, q[l], tabs[l].irp, tabs[l].ninv);
        else ntt_fwd_one(a, n, q[l], tabs[l].rp);
    }
    for (uint32_t l = 0; l < limbs; ++l) tab_free(&tabs[l]);
    free(tabs);
}

/* fast base conversion out_j = sum_i [x_i * qhat_i^-1]_{q_i} * [qhat_i]_{p_j} mod p_j
 * (src/rns_bconv.cu:109-210), with the products reduced exactly */
static void bconv(const uint64_t *x, const uint64_t *ib, uint32_t ni, const uint64_t *ob, uint32_t no,
                  uint64_t *const *out, uint32_t n) {
    uint64_t *qhat_inv = (uint64_t *)malloc(sizeof(uint64_t) * ni);
    uint64_t *qhat_mod = (uint64_t *)malloc(sizeof(uint64_t) * ni * no);
    for (uint32_t i = 0; i < ni; ++i) {
        uint64_t prod = 1;
        for (uint32_t k = 0; k < ni; ++k)
            if (k != i) prod = orc_mulmod(prod, ib[k] % ib[i], ib[i]);
        qhat_inv[i] = orc_invmod(prod, ib[i]);
        for (uint32_t j = 0; j < no; ++j) {
            uint64_t pm = 1 % ob[j];
            for (uint32_t k = 0; k < ni; ++k)
                if (k != i) pm = orc_mulmod(pm, ib[k] % ob[j], ob[j]);
            qhat_mod[(size_t)j * ni + i] = pm;
        }
    }
#pragma omp parallel for schedule(static)
    for (long c = 0; c < (long)n; ++c) {
        uint64_t y[64];
        for (uint32_t i = 0; i < ni; ++i) y[i] = orc_mulmod(x[(size_t)i * n + c], qhat_inv[i], ib[i]);
        for (uint32_t j = 0; j < no; ++j) {
            u128 acc = 0;
            for (uint32_t i = 0; i < ni; ++i) acc += (u128)y[i] * qhat_mod[(size_t)j * ni + i];
            out[j][c] = (uint64_t)(acc % ob[j]);
        }
    }
    free(qhat_mod);
    free(qhat_inv);
}

void orc_modup(const uint64_t *c2, uint64_t *out, uint32_t log_n, const uint64_t *q, uint32_t size_ql,
               const uint64_t *p, uint32_t size_p) {
    const uint32_t n = 1u << log_n, alpha = size_p, qlp = size_ql + size_p;
    const uint32_t beta = (size_ql + alpha - 1) / alpha;
    uint64_t *coef = (uint64_t *)malloc(sizeof(uint64_t) * size_ql * n);
    memcpy(coef, c2, sizeof(uint64_t) * size_ql * n);
    orc_rns_ntt(coef, 1, size_ql, log_n, q, 1);
    uint64_t *mods = (uint64_t *)malloc(sizeof(uint64_t) * qlp);
    for (uint32_t i = 0; i < size_ql; ++i) mods[i] = q[i];
    for (uint32_t j = 0; j < size_p; ++j) mods[size_ql + j] = p[j];
    for (uint32_t b = 0; b < beta; ++b) {
        const uint32_t start = alpha * b, cnt = (b == beta - 1) ? size_ql - alpha * (beta - 1) : alpha;
        uint64_t *blk = out + (size_t)b * qlp * n;
        /* own limbs: copied from the NTT-domain input */
        memcpy(blk + (size_t)start * n, c2 + (size_t)start * n, sizeof(uint64_t) * cnt * n);
        /* complement limbs: base conversion from the part, then NTT */
        uint32_t no = 0;
        uint64_t *ob = (uint64_t *)malloc(sizeof(uint64_t) * qlp);
        uint64_t **dst = (uint64_t **)malloc(sizeof(uint64_t *) * qlp);
        for (uint32_t l = 0; l < qlp; ++l)
            if (l < start || l >= start + cnt) {
                ob[no] = mods[l];
                dst[no++] = blk + (size_t)l * n;
            }
        bconv(coef + (size_t)start * n, q + start, cnt, ob, no, dst, n);
        for (uint32_t k = 0; k < no; ++k) {
            orc_tab t;
            tab_make(&t, log_n, ob[k]);
            ntt_fwd_one(dst[k], n, ob[k], t.rp);
            tab_free(&t);
        }
        free(dst);
        free(ob);
    }
    free(mods);
    free(coef);
}

void orc_ks_inner(const uint64_t *t, const uint64_t *evk, uint64_t *cx, uint32_t n, const uint64_t *q, uint32_t size_ql,
                  uint32_t size_q, const uint64_t *p, uint32_t size_p) {
    const uint32_t alpha = size_p, qlp = size_ql + size_p, qp = size_q + size_p;
    const uint32_t beta = (size_ql + alpha - 1) / alpha;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < (long)qlp; ++l) {
        const uint64_t m = (l < (long)size_ql) ? q[l] : p[l - size_ql];
        const uint32_t kl = (l < (long)size_ql) ? (uint32_t)l : size_q + (uint32_t)(l - size_ql);
        for (uint32_t c = 0; c < n; ++c) {
            u128 a0 = 0, a1 = 0;
            for (uint32_t b = 0; b < beta; ++b) {
                const uint64_t x = t[((size_t)b * qlp + l) * n + c];
                const uint64_t *ek = evk + (size_t)b * 2 * qp * n;
                a0 += (u128)x * ek[(size_t)kl * n + c];
                a1 += (u128)x * ek[(size_t)(qp + kl) * n + c];
            }
            cx[(size_t)l * n + c] = (uint64_t)(a0 % m);
            cx[((size_t)qlp + l) * n + c] = (uint64_t)(a1 % m);
        }
    }
}

void orc_moddown(const uint64_t *cx, uint64_t *ct, uint32_t log_n, const uint64_t *q, uint32_t size_ql,
                 const uint64_t *p, uint32_t size_p) {
    const uint32_t n = 1u << log_n;
    uint64_t *cp = (uint64_t *)malloc(sizeof(uint64_t) * size_p * n);
    memcpy(cp, cx + (size_t)size_ql * n, sizeof(uint64_t) * size_p * n);
    orc_rns_ntt(cp, 1, size_p, log_n, p, 1);
    uint64_t *delta = (uint64_t *)malloc(sizeof(uint64_t) * size_ql * n);
    uint64_t **dst = (uint64_t **)malloc(sizeof(uint64_t *) * size_ql);
    for (uint32_t i = 0; i < size_ql; ++i) dst[i] = delta + (size_t)i * n;
    bconv(cp, p, size_p, q, size_ql, dst, n);
    orc_rns_ntt(delta, 1, size_ql, log_n, q, 0);
    for (uint32_t i = 0; i < size_ql; ++i) {
        uint64_t P = 1;
        for (uint32_t k = 0; k < size_p; ++k) P = orc_mulmod(P, p[k] % q[i], q[i]);
        const uint64_t pinv = orc_invmod(P, q[i]);
        for (uint32_t c = 0; c < n; ++c)
            ct[(size_t)i * n + c] =
                orc_mulmod(submod(cx[(size_t)i * n + c], delta[(size_t)i * n + c], q[i]), pinv, q[i]);
    }
    free(dst);
    free(delta);
    free(cp);
}

void orc_keyswitch(uint64_t *ct, const uint64_t *c2, const uint64_t *evk, uint32_t log_n, const uint64_t *q,
                   uint32_t size_ql, uint32_t size_q, const uint64_t *p, uint32_t size_p) {
    const uint32_t n = 1u << log_n, alpha = size_p, qlp = size_ql + size_p;
    const uint32_t beta = (size_ql + alpha - 1) / alpha;
    uint64_t *t = (uint64_t *)malloc(sizeof(uint64_t) * beta * qlp * n);
    uint64_t *cx = (uint64_t *)malloc(sizeof(uint64_t) * 2 * qlp * n);
    uint64_t *d = (uint64_t *)malloc(sizeof(uint64_t) * size_ql * n);
    orc_modup(c2, t, log_n, q, size_ql, p, size_p);
    orc_ks_inner(t, evk, cx, n, q, size_ql, size_q, p, size_p);
    for (uint32_t k = 0; k < 2; ++k) {
        orc_moddown(cx + (size_t)k * qlp * n, d, log_n, q, size_ql, p, size_p);
        for (uint32_t i = 0; i < size_ql; ++i)
            for (uint32_t c = 0; c < n; ++c) {
                uint64_t *dst = ct + ((size_t)k * size_ql + i) * n + c;
                *dst = addmod(*dst, d[(size_t)i * n + c], q[i]);
            }
    }
    free(d);
    free(cx);
    free(t);
}

/* ------------------------------------------------------------------------------------------ */
/* gate bootstrap on the 32-bit torus                                                          */
/* ------------------------------------------------------------------------------------------ */

void orc_gate_combine(int gate, const uint32_t *a1, uint32_t b1, const uint32_t *a2, uint32_t b2, uint32_t n,
                      uint32_t *a, uint32_t *b) {
    const uint32_t e8 = 1u << 29, e4 = 1u << 30; /* 1/8, 1/4 */
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t s = a1[i] + a2[i];
        switch (gate) {
            case 0: case 1: a[i] = s; break;         /* OR, AND: + c1 + c2 */
            case 2: case 3: a[i] = 0u - s; break;    /* NOR, NAND: - c1 - c2 */
            case 4: a[i] = 2u * s; break;            /* XOR: 2 (c1 + c2) */
            default: a[i] = 0u - 2u * s; break;      /* XNOR: -2 (c1 + c2) */
        }
    }
    const uint32_t s = b1 + b2;
    switch (gate) {
        case 0: *b = e8 + s; break;
        case 1: *b = (0u - e8) + s; break;
        case 2: *b = (0u - e8) - s; break;
        case 3: *b = e8 - s; break;
        case 4: *b = e4 + 2u * s; break;
        default: *b = (0u - e4) - 2u * s; break;
    }
}

/* acc += X^e * src (negacyclic, mod 2^32) */
static void torus_rot_add(uint32_t *acc, const uint32_t *src, uint32_t e, uint32_t N) {
    for (uint32_t i = 0; i < N; ++i) {
        uint32_t t = (i + e) % (2 * N);
        if (t < N) acc[t] += src[i];
        else acc[t - N] -= src[i];
    }
}

/* out += d * k (negacyclic, d small signed digits, k torus32) */
static void torus_mac(uint32_t *out, const int32_t *d, const uint32_t *k, uint32_t N) {
    for (uint32_t i = 0; i < N; ++i) {
        if (!d[i]) continue;
        const uint32_t di = (uint32_t)d[i];
        for (uint32_t j = 0; j < N; ++j) {
            const uint32_t v = di * k[j];
            if (i + j < N) out[i + j] += v;
            else out[i + j - N] -= v;
        }
    }
}

/* signed base-2^bg digits, most significant first, of the top bg*levels bits (rounded) */
static void torus_decompose(uint32_t x, uint32_t bg_bits, uint32_t levels, int32_t *d) {
    uint32_t off = 0;
    for (uint32_t k = 0; k < levels; ++k) off += (1u << (bg_bits - 1)) << (32 - (k + 1) * bg_bits);
    off += 1u << (32 - levels * bg_bits - 1);
    const uint32_t w = x + off;
    for (uint32_t k = 0; k < levels; ++k)
        d[k] = (int32_t)((w >> (32 - (k + 1) * bg_bits)) & ((1u << bg_bits) - 1)) - (int32_t)(1u << (bg_bits - 1));
}

void orc_gate_blind_rotate(const orc_gate_params *p, const uint32_t *bsk, const uint32_t *a, uint32_t b,
                           uint32_t *ext) {
    orc_gate_blind_rotate_tv(p, bsk, a, b, 1u << 29, 0, ext);
}

void orc_gate_blind_rotate_tv(const orc_gate_params *p, const uint32_t *bsk, const uint32_t *a, uint32_t b,
                              uint32_t mu, uint32_t b_add, uint32_t *ext) {
    orc_gate_blind_rotate_lut(p, bsk, a, b, NULL, mu, b_add, ext);
}

/* the same rotation of an arbitrary test vector tv [N] (coefficient domain; NULL: the constant mu) */
void orc_gate_blind_rotate_lut(const orc_gate_params *p, const uint32_t *bsk, const uint32_t *a, uint32_t b,
                               const uint32_t *tv, uint32_t mu, uint32_t b_add, uint32_t *ext) {
    const uint32_t N = p->N, L = p->levels, two_n = 2 * N;
    uint32_t logn2 = 0;
    while ((1u << logn2) < two_n) ++logn2;
    const uint32_t sh = 32 - logn2;
#define MS(x) ((uint32_t)(((x) + (1u << (sh - 1))) >> sh) & (two_n - 1))
    uint32_t *acc = (uint32_t *)calloc(2 * N, sizeof(uint32_t));
    uint32_t *prod = (uint32_t *)malloc(2 * N * sizeof(uint32_t));
    int32_t *dig = (int32_t *)malloc((size_t)2 * L * N * sizeof(int32_t));
    /* acc = (0, X^-b~ * TV), TV = 1/8 everywhere */
    const uint32_t bt = MS(b);
    for (uint32_t i = 0; i < N; ++i) {
        const uint32_t s = (i + bt) % two_n; /* coefficient i of X^-bt TV = TV[i + bt] (wrapped) */
        const uint32_t v = tv ? tv[s % N] : mu;
        acc[N + i] = (s < N) ? v : 0u - v;
    }
    for (uint32_t step = 0; step < p->n; ++step) {
        const uint32_t at = MS(a[step]);
        if (at == 0) continue;
        int32_t dd[8];
        for (uint32_t c = 0; c < 2; ++c)
            for (uint32_t i = 0; i < N; ++i) {
                torus_decompose(acc[c * N + i], p->bg_bits, L, dd);
                for (uint32_t k = 0; k < L; ++k) dig[((size_t)(2 * k + c)) * N + i] = dd[k];
            }
        memset(prod, 0, 2 * N * sizeof(uint32_t));
        const uint32_t *key = bsk + (size_t)step * 2 * L * 2 * N;
        for (uint32_t r = 0; r < 2 * L; ++r)
            for (uint32_t c = 0; c < 2; ++c)
                torus_mac(prod + c * N, dig + (size_t)r * N, key + ((size_t)r * 2 + c) * N, N);
        for (uint32_t c = 0; c < 2; ++c) {
            torus_rot_add(acc + c * N, prod + c * N, at, N);
            for (uint32_t i = 0; i < N; ++i) acc[c * N + i] -= prod[c * N + i];
        }
    }
#undef MS
    /* sample extract of coefficient 0 */
    ext[0] = acc[0];
    for (uint32_t i = 1; i < N; ++i) ext[i] = 0u - acc[N - i];
    ext[N] = acc[N] + b_add;
    free(dig);
    free(prod);
    free(acc);
}

/* out += d * k (negacyclic, d small signed digits, k torus64) */
static void torus64_mac(uint64_t *out, const int32_t *d, const uint64_t *k, uint32_t N) {
    for (uint32_t i = 0; i < N; ++i) {
        if (!d[i]) continue;
        const uint64_t di = (uint64_t)(int64_t)d[i];
        for (uint32_t j = 0; j < N; ++j) {
            const uint64_t v = di * k[j];
            if (i + j < N) out[i + j] += v;
            else out[i + j - N] -= v;
        }
    }
}

void orc_tcb_blind_rotate64(const orc_gate_params *p, const uint64_t *bsk, const uint32_t *a, uint32_t b,
                            uint64_t mu, uint64_t b_add, uint64_t *ext) {
    const uint32_t N = p->N, L = p->levels, two_n = 2 * N, bg = p->bg_bits;
    uint32_t logn2 = 0;
    while ((1u << logn2) < two_n) ++logn2;
    const uint32_t sh = 32 - logn2;
#define MS(x) ((uint32_t)(((x) + (1u << (sh - 1))) >> sh) & (two_n - 1))
    uint64_t *acc = (uint64_t *)calloc(2 * N, sizeof(uint64_t));
    uint64_t *prod = (uint64_t *)malloc(2 * N * sizeof(uint64_t));
    int32_t *dig = (int32_t *)malloc((size_t)2 * L * N * sizeof(int32_t));
    uint64_t off = 1ull << (64 - L * bg - 1);
    for (uint32_t k = 0; k < L; ++k) off += (1ull << (bg - 1)) << (64 - (k + 1) * bg);
    const uint32_t bt = MS(b);
    for (uint32_t i = 0; i < N; ++i) acc[N + i] = ((i + bt) % two_n < N) ? mu : 0ull - mu;
    for (uint32_t step = 0; step < p->n; ++step) {
        const uint32_t at = MS(a[step]);
        if (at == 0) continue;
        for (uint32_t c = 0; c < 2; ++c)
            for (uint32_t i = 0; i < N; ++i) {
                const uint64_t w = acc[c * N + i] + off;
                for (uint32_t k = 0; k < L; ++k)
                    dig[((size_t)(2 * k + c)) * N + i] =
                        (int32_t)((w >> (64 - (k + 1) * bg)) & ((1u << bg) - 1)) - (int32_t)(1u << (bg - 1));
            }
        memset(prod, 0, 2 * N * sizeof(uint64_t));
        const uint64_t *key = bsk + (size_t)step * 2 * L * 2 * N;
        for (uint32_t r = 0; r < 2 * L; ++r)
            for (uint32_t c = 0; c < 2; ++c)
                torus64_mac(prod + c * N, dig + (size_t)r * N, key + ((size_t)r * 2 + c) * N, N);
        for (uint32_t c = 0; c < 2; ++c)
            for (uint32_t i = 0; i < N; ++i) {
                const uint32_t t = (i + at) % two_n;
                if (t < N) acc[c * N + t] += prod[c * N + i];
                else acc[c * N + t - N] -= prod[c * N + i];
                acc[c * N + i] -= prod[c * N + i];
            }
    }
#undef MS
    ext[0] = acc[0];
    for (uint32_t i = 1; i < N; ++i) ext[i] = 0ull - acc[N - i];
    ext[N] = acc[N] + b_add;
    free(dig);
    free(prod);
    free(acc);
}

/* Multi-bit (grouped) forms of the two torus blind rotations above, the reference's
 * CIRBTS_PBS_MULTIBIT grouping (cirbts-init.cu:376-530, kernel.cu:4585-4771) on the torus:
 * per group of mb coefficients, acc += sum_S m_S (acc (x) RGSW(prod_{i in S} s_i)) with
 * m_S = prod_{i in S} (X^{a_i} - 1), subsets in the order of orc_mb_order2 / orc_mb_order3.
 * mbk [ceil(n/mb)][2^mb - 1][2*levels][2][N].  Groups whose rotations are all 0 add nothing
 * and are skipped. */
static void torus_mono_minus1(uint32_t *p, uint32_t e, uint32_t N, uint32_t *tmp) {
    memset(tmp, 0, N * sizeof(uint32_t));
    torus_rot_add(tmp, p, e, N);
    for (uint32_t i = 0; i < N; ++i) p[i] = tmp[i] - p[i];
}

void orc_gate_blind_rotate_tv_mb(const orc_gate_params *p, const uint32_t *mbk, uint32_t mb, const uint32_t *a,
                                 uint32_t b, uint32_t mu, uint32_t b_add, uint32_t *ext) {
    const uint32_t N = p->N, L = p->levels, two_n = 2 * N, K = (1u << mb) - 1u;
    const uint32_t groups = (p->n + mb - 1) / mb;
    const uint32_t *order = (mb == 2) ? orc_mb_order2 : orc_mb_order3;
    uint32_t logn2 = 0;
    while ((1u << logn2) < two_n) ++logn2;
    const uint32_t sh = 32 - logn2;
#define MS(x) ((uint32_t)(((x) + (1u << (sh - 1))) >> sh) & (two_n - 1))
    uint32_t *acc = (uint32_t *)calloc(2 * N, sizeof(uint32_t));
    uint32_t *prod = (uint32_t *)malloc(2 * N * sizeof(uint32_t));
    uint32_t *tmp = (uint32_t *)malloc(N * sizeof(uint32_t));
    int32_t *dig = (int32_t *)malloc((size_t)2 * L * N * sizeof(int32_t));
    const uint32_t bt = MS(b);
    for (uint32_t i = 0; i < N; ++i) acc[N + i] = ((i + bt) % two_n < N) ? mu : 0u - mu;
    for (uint32_t g = 0; g < groups; ++g) {
        uint32_t at[3] = {0, 0, 0}, any = 0;
        for (uint32_t i = 0; i < mb; ++i) {
            const uint32_t idx = g * mb + i;
            at[i] = idx < p->n ? MS(a[idx]) : 0u;
            any |= at[i];
        }
        if (!any) continue;
        int32_t dd[8];
        for (uint32_t c = 0; c < 2; ++c)
            for (uint32_t i = 0; i < N; ++i) {
                torus_decompose(acc[c * N + i], p->bg_bits, L, dd);
                for (uint32_t k = 0; k < L; ++k) dig[((size_t)(2 * k + c)) * N + i] = dd[k];
            }
        for (uint32_t kk = 0; kk < K; ++kk) {
            memset(prod, 0, 2 * N * sizeof(uint32_t));
            const uint32_t *key = mbk + ((size_t)g * K + kk) * 2 * L * 2 * N;
            for (uint32_t r = 0; r < 2 * L; ++r)
                for (uint32_t c = 0; c < 2; ++c)
                    torus_mac(prod + c * N, dig + (size_t)r * N, key + ((size_t)r * 2 + c) * N, N);
            for (uint32_t i = 0; i < mb; ++i)
                if (order[kk] & (1u << i))
                    for (uint32_t c = 0; c < 2; ++c) torus_mono_minus1(prod + c * N, at[i], N, tmp);
            for (uint32_t j = 0; j < 2 * N; ++j) acc[j] += prod[j];
        }
    }
#undef MS
    ext[0] = acc[0];
    for (uint32_t i = 1; i < N; ++i) ext[i] = 0u - acc[N - i];
    ext[N] = acc[N] + b_add;
    free(dig);
    free(tmp);
    free(prod);
    free(acc);
}

static void torus64_mono_minus1(uint64_t *p, uint32_t e, uint32_t N, uint64_t *tmp) {
    memset(tmp, 0, N * sizeof(uint64_t));
    for (uint32_t i = 0; i < N; ++i) {
        const uint32_t t = (i + e) % (2 * N);
        if (t < N) tmp[t] += p[i];
        else tmp[t - N] -= p[i];
    }
    for (uint32_t i = 0; i < N; ++i) p[i] = tmp[i] - p[i];
}

void orc_tcb_blind_rotate64_mb(const orc_gate_params *p, const uint64_t *mbk, uint32_t mb, const uint32_t *a,
                               uint32_t b, uint64_t mu, uint64_t b_add, uint64_t *ext) {
    const uint32_t N = p->N, L = p->levels, two_n = 2 * N, bg = p->bg_bits, K = (1u << mb) - 1u;
    const uint32_t groups = (p->n + mb - 1) / mb;
    const uint32_t *order = (mb == 2) ? orc_mb_order2 : orc_mb_order3;
    uint32_t logn2 = 0;
    while ((1u << logn2) < two_n) ++logn2;
    const uint32_t sh = 32 - logn2;
#define MS(x) ((uint32_t)(((x) + (1u << (sh - 1))) >> sh) & (two_n - 1))
    uint64_t *acc = (uint64_t *)calloc(2 * N, sizeof(uint64_t));
    uint64_t *prod = (uint64_t *)malloc(2 * N * sizeof(uint64_t));
    uint64_t *tmp = (uint64_t *)malloc(N * sizeof(uint64_t));
    int32_t *dig = (int32_t *)malloc((size_t)2 * L * N * sizeof(int32_t));
    uint64_t off = 1ull << (64 - L * bg - 1);
    for (uint32_t k = 0; k < L; ++k) off += (1ull << (bg - 1)) << (64 - (k + 1) * bg);
    const uint32_t bt = MS(b);
    for (uint32_t i = 0; i < N; ++i) acc[N + i] = ((i + bt) % two_n < N) ? mu : 0ull - mu;
    for (uint32_t g = 0; g < groups; ++g) {
        uint32_t at[3] = {0, 0, 0}, any = 0;
        for (uint32_t i = 0; i < mb; ++i) {
            const uint32_t idx = g * mb + i;
            at[i] = idx < p->n ? MS(a[idx]) : 0u;
            any |= at[i];
        }
        if (!any) continue;
        for (uint32_t c = 0; c < 2; ++c)
            for (uint32_t i = 0; i < N; ++i) {
                const uint64_t w = acc[c * N + i] + off;
                for (uint32_t k = 0; k < L; ++k)
                    dig[((size_t)(2 * k + c)) * N + i] =
                        (int32_t)((w >> (64 - (k + 1) * bg)) & ((1u << bg) - 1)) - (int32_t)(1u << (bg - 1));
            }
        for (uint32_t kk = 0; kk < K; ++kk) {
            memset(prod, 0, 2 * N * sizeof(uint64_t));
            const uint64_t *key = mbk + ((size_t)g * K + kk) * 2 * L * 2 * N;
            for (uint32_t r = 0; r < 2 * L; ++r)
                for (uint32_t c = 0; c < 2; ++c)
                    torus64_mac(prod + c * N, dig + (size_t)r * N, key + ((size_t)r * 2 + c) * N, N);
            for (uint32_t i = 0; i < mb; ++i)
                if (order[kk] & (1u << i))
                    for (uint32_t c = 0; c < 2; ++c) torus64_mono_minus1(prod + c * N, at[i], N, tmp);
            for (uint32_t j = 0; j < 2 * N; ++j) acc[j] += prod[j];
        }
    }
#undef MS
    ext[0] = acc[0];
    for (uint32_t i = 1; i < N; ++i) ext[i] = 0ull - acc[N - i];
    ext[N] = acc[N] + b_add;
    free(dig);
    free(tmp);
    free(prod);
    free(acc);
}

void orc_tcb_pfks(uint32_t N2, uint32_t N1, uint32_t base_bits, uint32_t levels, const uint32_t *key,
                  const uint64_t *ext, uint32_t *out) {
    const uint32_t base = 1u << base_bits;
    memset(out, 0, 2 * N1 * sizeof(uint32_t));
    for (uint32_t i = 0; i <= N2; ++i) {
        const uint64_t x64 = (i < N2) ? 0ull - ext[i] : ext[N2]; /* phase = sum x_i y_i */
        const uint32_t x = (uint32_t)((x64 + (1ull << 31)) >> 32);  /* top 32 bits, rounded */
        for (uint32_t j = 0; j < levels; ++j) {
            const uint32_t v = (x >> (32 - (j + 1) * base_bits)) & (base - 1);
            if (!v) continue;
            const uint32_t *row = key + (((size_t)i * levels + j) * (base - 1) + (v - 1)) * 2 * N1;
            for (uint32_t c = 0; c < 2 * N1; ++c) out[c] += row[c];
        }
    }
}

void orc_gate_keyswitch(const orc_gate_params *p, const uint32_t *ksk, const uint32_t *ext, uint32_t *out) {
    const uint32_t N = p->N, n = p->n, t = p->ks_levels, bb = p->ks_base_bits, base = 1u << bb;
    const uint32_t round = 1u << (32 - t * bb - 1);
    for (uint32_t j = 0; j <= n; ++j) out[j] = 0;
    out[n] = ext[N];
    for (uint32_t i = 0; i < N; ++i) {
        const uint32_t x = ext[i] + round;
        for (uint32_t l = 0; l < t; ++l) {
            const uint32_t v = (x >> (32 - (l + 1) * bb)) & (base - 1);
            if (!v) continue;
            const uint32_t *row = ksk + (((size_t)i * t + l) * (base - 1) + (v - 1)) * (n + 1);
            for (uint32_t j = 0; j <= n; ++j) out[j] -= row[j];
        }
    }
}

/* the programmable bootstrap of the functional evaluators (binfhe-base-scheme-batch.cu:215-364):
 * a [n], b mod 2^in_bits lifted to the torus, the test vector (2^32 / 2^f_bits) lut[j] at
 * coefficient j 2N / 2^in_bits (j < 2^in_bits / 2), rotation, extraction, key switch to n, and the
 * rounding to Z_(2^f_bits).  out [n + 1] (a then b). */
void orc_gate_bootstrap_func(const orc_gate_params *p, const uint32_t *bsk, const uint32_t *ksk, const uint32_t *a,
                             uint32_t b, uint32_t in_bits, const uint64_t *lut, uint32_t f_bits, uint32_t *out) {
    const uint32_t N = p->N, n = p->n, q_in = 1u << in_bits, factor = 2 * N / q_in;
    uint32_t *tv = (uint32_t *)calloc(N, sizeof(uint32_t));
    uint32_t *at = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint32_t *ext = (uint32_t *)malloc(sizeof(uint32_t) * (N + 1));
    for (uint32_t j = 0; j < q_in / 2; ++j) tv[j * factor] = (uint32_t)(lut[j] << (32 - f_bits));
    for (uint32_t i = 0; i < n; ++i) at[i] = a[i] << (32 - in_bits);
    orc_gate_blind_rotate_lut(p, bsk, at, b << (32 - in_bits), tv, 0, 0, ext);
    orc_gate_keyswitch(p, ksk, ext, out);
    const uint32_t sh = 32 - f_bits, mask = f_bits >= 32 ? ~0u : ((1u << f_bits) - 1u);
    for (uint32_t i = 0; i <= n; ++i) {
        const uint64_t x = out[i];
        out[i] = (uint32_t)(sh ? (x + (1ull << (sh - 1))) >> sh : x) & mask;
    }
    free(ext);
    free(at);
    free(tv);
}

/* ------------------------------------------------------------------------------------------ */
/* plaintext AES-128 (FIPS-197), restating examples/aes_transcipher/aes128.cuh                 */
/* ------------------------------------------------------------------------------------------ */

static uint8_t gmul(uint8_t a, uint8_t b) {
    uint8_t p = 0;
    while (b) {
        if (b & 1) p ^= a;
        a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1b : 0));
        b >>= 1;
    }
    return p;
}

/* S-box from its definition: multiplicative inverse in GF(2^8) followed by the affine map */
static void build_sbox(uint8_t sbox[256]) {
    for (int x = 0; x < 256; ++x) {
        uint8_t inv = 0;
        if (x) {
            for (int y = 1; y < 256; ++y)
                if (gmul((uint8_t)x, (uint8_t)y) == 1) { inv = (uint8_t)y; break; }
        }
        uint8_t s = inv;
        for (int i = 1; i <= 4; ++i) s ^= (uint8_t)((inv << i) | (inv >> (8 - i)));
        sbox[x] = (uint8_t)(s ^ 0x63);
    }
}

static const uint8_t *get_sbox(void) {
    static uint8_t sbox[256];
    static int ready = 0;
    if (!ready) {
#pragma omp critical(orc_sbox)
        {
            if (!ready) { build_sbox(sbox); ready = 1; }
        }
    }
    return sbox;
}

/* aes128.cuh:99-121 Aes128KeyExpand; round_keys[r][i] in column-major state order */
void orc_aes128_key_expand(const uint8_t key[16], uint8_t rk[11][16]) {
    const uint8_t *sbox = get_sbox();
    uint8_t w[44][4];
    static const uint8_t rcon[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) w[i][j] = key[4 * i + j];
    for (int i = 4; i < 44; ++i) {
        uint8_t t[4] = {w[i - 1][0], w[i - 1][1], w[i - 1][2], w[i - 1][3]};
        if (i % 4 == 0) {
            const uint8_t t0 = t[0];
            t[0] = (uint8_t)(sbox[t[1]] ^ rcon[i / 4 - 1]);
            t[1] = sbox[t[2]];
            t[2] = sbox[t[3]];
            t[3] = sbox[t0];
        }
        for (int j = 0; j < 4; ++j) w[i][j] = (uint8_t)(w[i - 4][j] ^ t[j]);
    }
    for (int r = 0; r < 11; ++r)
        for (int c = 0; c < 4; ++c)
            for (int row = 0; row < 4; ++row) rk[r][c * 4 + row] = w[r * 4 + c][row];
}

/* aes128.cuh:151-165 Aes128EncryptPlain */
void orc_aes128_encrypt(const uint8_t key[16], const uint8_t in[16], uint8_t out[16]) {
    const uint8_t *sbox = get_sbox();
    uint8_t rk[11][16], s[16], t[16];
    orc_aes128_key_expand(key, rk);
    for (int i = 0; i < 16; ++i) s[i] = in[i] ^ rk[0][i];
    for (int r = 1; r <= 10; ++r) {
        for (int i = 0; i < 16; ++i) s[i] = sbox[s[i]];
        for (int row = 0; row < 4; ++row)
            for (int c = 0; c < 4; ++c) t[c * 4 + row] = s[((c + row) & 3) * 4 + row];
        memcpy(s, t, 16);
        if (r != 10) {
            for (int c = 0; c < 4; ++c) {
                const uint8_t a0 = s[c * 4], a1 = s[c * 4 + 1], a2 = s[c * 4 + 2], a3 = s[c * 4 + 3];
                s[c * 4 + 0] = (uint8_t)(gmul(a0, 2) ^ gmul(a1, 3) ^ a2 ^ a3);
                s[c * 4 + 1] = (uint8_t)(a0 ^ gmul(a1, 2) ^ gmul(a2, 3) ^ a3);
                s[c * 4 + 2] = (uint8_t)(a0 ^ a1 ^ gmul(a2, 2) ^ gmul(a3, 3));
                s[c * 4 + 3] = (uint8_t)(gmul(a0, 3) ^ a1 ^ a2 ^ gmul(a3, 2));
            }
        }
        for (int i = 0; i < 16; ++i) s[i] ^= rk[r][i];
    }
    memcpy(out, s, 16);
}

static uint32_t pack_be(uint8_t b0, uint8_t b1, uint8_t b2, uint8_t b3) {
    return ((uint32_t)b0 << 24) | ((uint32_t)b1 << 16) | ((uint32_t)b2 << 8) | b3;
}
static uint32_t rotr(uint32_t x, int r) { return (x >> r) | (x << (32 - r)); }

/* aes128.cuh:316-330 BuildAesEncTables */
void orc_aes_enc_tables(uint32_t te[8][256]) {
    const uint8_t *sbox = get_sbox();
    for (int x = 0; x < 256; ++x) {
        const uint8_t s = sbox[x];
        const uint32_t t0 = pack_be(gmul(s, 2), s, s, gmul(s, 3));
        te[0][x] = t0;
        te[1][x] = rotr(t0, 8);
        te[2][x] = rotr(t0, 16);
        te[3][x] = rotr(t0, 24);
        te[4][x] = pack_be(s, 0, 0, 0);
        te[5][x] = pack_be(0, s, 0, 0);
        te[6][x] = pack_be(0, 0, s, 0);
        te[7][x] = pack_be(0, 0, 0, s);
    }
}


/* ---------------- encryption of the AES material ---------------- */

static uint32_t orc_rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

static void orc_chacha_qr(uint32_t *x, int a, int b, int c, int d) {
    x[a] += x[b]; x[d] = orc_rotl32(x[d] ^ x[a], 16);
    x[c] += x[d]; x[b] = orc_rotl32(x[b] ^ x[c], 12);
    x[a] += x[b]; x[d] = orc_rotl32(x[d] ^ x[a], 8);
    x[c] += x[d]; x[b] = orc_rotl32(x[b] ^ x[c], 7);
}

void orc_chacha20_block(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3], uint32_t out[16]) {
    uint32_t in[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
    for (int i = 0; i < 8; ++i) in[4 + i] = key[i];
    in[12] = counter;
    in[13] = nonce[0];
    in[14] = nonce[1];
    in[15] = nonce[2];
    uint32_t x[16];
    memcpy(x, in, sizeof(x));
    for (int r = 0; r < 10; ++r) {
        orc_chacha_qr(x, 0, 4, 8, 12);
        orc_chacha_qr(x, 1, 5, 9, 13);
        orc_chacha_qr(x, 2, 6, 10, 14);
        orc_chacha_qr(x, 3, 7, 11, 15);
        orc_chacha_qr(x, 0, 5, 10, 15);
        orc_chacha_qr(x, 1, 6, 11, 12);
        orc_chacha_qr(x, 2, 7, 8, 13);
        orc_chacha_qr(x, 3, 4, 9, 14);
    }
    for (int i = 0; i < 16; ++i) out[i] = x[i] + in[i];
}

uint64_t orc_uniform_mod(const uint32_t w[4], uint64_t q) {
    const u128 x = (u128)w[0] | ((u128)w[1] << 32) | ((u128)w[2] << 64) | ((u128)w[3] << 96);
    /* floor(x q / 2^128) = floor((hi q + floor(lo q / 2^64)) / 2^64) */
    const uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
    const u128 t = (u128)hi * q + (uint64_t)(((u128)lo * q) >> 64);
    return (uint64_t)(t >> 64);
}

uint32_t orc_cdt_table(double sigma, uint64_t *T, uint32_t cap) {
    if (!(sigma > 0)) return 0;
    const long double s2 = 2.0L * (long double)sigma * (long double)sigma;
    const int X = (int)ceil(14.0 * sigma) + 1;
    long double S = 1.0L;
    for (int x = 1; x <= X; ++x) S += 2.0L * expl(-(long double)x * x / s2);
    const long double two63 = 9223372036854775808.0L;
    long double cum = 1.0L;
    uint32_t len = 0;
    for (int k = 0; k <= X; ++k) {
        if (k > 0) cum += 2.0L * expl(-(long double)k * k / s2);
        const long double t = floorl(two63 * (cum / S));
        if (t >= two63) break;
        if (len < cap) T[len] = (uint64_t)t;
        ++len;
    }
    return len;
}

int64_t orc_cdt_sample(uint64_t u, const uint64_t *T, uint32_t len) {
    const uint64_t v = u & 0x7fffffffffffffffull;
    int64_t mag = 0;
    for (uint32_t k = 0; k < len; ++k) mag += v >= T[k];
    return (u >> 63) ? -mag : mag;
}

void orc_encrypt_words_rlwe(const uint32_t key[8], const uint32_t *words, uint32_t count, uint32_t first, uint32_t N,
                            uint64_t Q, const uint64_t *rp, const uint64_t *s_ntt, const uint64_t *T, uint32_t tlen,
                            uint64_t *out) {
    uint64_t *tmp = (uint64_t *)malloc((size_t)N * sizeof(uint64_t));
    for (uint32_t r = 0; r < count; ++r) {
        uint64_t *a = out + (size_t)r * 2 * N, *b = a + N;
        const uint32_t nonce[3] = {first + r, 1u, 0u};
        for (uint32_t i = 0; i < N; ++i) {
            uint32_t blk[16];
            orc_chacha20_block(key, i, nonce, blk);
            a[i] = orc_uniform_mod(blk, Q);
            const int64_t e = orc_cdt_sample((uint64_t)blk[4] | ((uint64_t)blk[5] << 32), T, tlen);
            uint64_t v = e < 0 ? Q - (uint64_t)(-e) : (uint64_t)e;
            if (i < 32 && ((words[r] >> i) & 1u)) v = (v + (Q >> 1)) % Q;
            tmp[i] = v;
        }
        orc_ntt_forward(tmp, 1, N, Q, rp);
        for (uint32_t i = 0; i < N; ++i) b[i] = (orc_mulmod(a[i], s_ntt[i], Q) + tmp[i]) % Q;
    }
    free(tmp);
}

void orc_encrypt_bits_lwe(const uint32_t key[8], const uint8_t *bits, uint32_t count, uint32_t n, uint64_t q,
                          const int32_t *s, const uint64_t *T, uint32_t tlen, uint64_t *a, uint64_t *b) {
    for (uint32_t t = 0; t < count; ++t) {
        const uint32_t nonce[3] = {t, 2u, 0u};
        u128 acc = 0;
        uint32_t blk[16];
        for (uint32_t i = 0; i < n; ++i) {
            orc_chacha20_block(key, i, nonce, blk);
            a[(size_t)t * n + i] = orc_uniform_mod(blk, q);
            if (s[i]) acc += a[(size_t)t * n + i];
        }
        orc_chacha20_block(key, n, nonce, blk);
        const int64_t e = orc_cdt_sample((uint64_t)blk[4] | ((uint64_t)blk[5] << 32), T, tlen);
        const uint64_t eq = e < 0 ? q - (uint64_t)(-e) % q : (uint64_t)e % q;
        b[t] = (uint64_t)((acc % q + (bits[t] ? q >> 1 : 0) + eq) % q);
    }
}

/* ------------------------------------------------------------------------------------------ */
/* key generation for the CPU legs (restates the CUDA path's seeded host key generation)       */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    uint64_t s[4];
} orc_rng;

static uint64_t rng_splitmix(uint64_t *x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static void rng_seed(orc_rng *r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) r->s[i] = rng_splitmix(&x);
}

/* xoshiro256** */
static uint64_t rng_next(orc_rng *r) {
    uint64_t *s = r->s;
    const uint64_t m = s[1] * 5;
    const uint64_t out = ((m << 7) | (m >> 57)) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
    return out;
}

/* uniform below bound: rejection on the smallest covering bit mask */
static uint64_t rng_uniform(orc_rng *r, uint64_t bound) {
    int bits = 0;
    while (bits < 64 && ((bound - 1) >> bits)) ++bits;
    const uint64_t mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    for (;;) {
        const uint64_t v = rng_next(r) & mask;
        if (v < bound) return v;
    }
}

static int64_t rng_rounded_gaussian(orc_rng *r, double sigma) {
    const double u1 = ((double)(rng_next(r) >> 11) + 1.0) * 0x1.0p-53;
    const double u2 = (double)(rng_next(r) >> 11) * 0x1.0p-53;
    const double g = sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
    return (int64_t)llround(g * sigma);
}

static uint64_t mod_signed(int64_t v, uint64_t q) {
    const int64_t m = v % (int64_t)q;
    return m < 0 ? (uint64_t)(m + (int64_t)q) : (uint64_t)m;
}

/* gadget g_j = 2^(ign + j gbits), ign = log2 Q - digits gbits (kernel.cu:37-68) */
static void gadget_powers(uint64_t Q, uint32_t base, uint32_t digits, uint64_t *g) {
    const int gb = __builtin_ctz(base);
    const int logq = 64 - __builtin_clzll(Q);
    int ign = logq - (int)digits * gb;
    if (ign < 0) ign = 0;
    for (uint32_t j = 0; j < digits; ++j) g[j] = (1ull << (ign + (int)j * gb)) % Q;
}

/* a uniform (NTT domain), b = a s + NTT(e) */
static void keygen_rlwe_zero(orc_rng *r, uint32_t N, uint64_t Q, double sigma, const uint64_t *rp,
                             const uint64_t *s_ntt, uint64_t *a, uint64_t *b, uint64_t *tmp) {
    for (uint32_t i = 0; i < N; ++i) a[i] = rng_uniform(r, Q);
    for (uint32_t i = 0; i < N; ++i) tmp[i] = mod_signed(rng_rounded_gaussian(r, sigma), Q);
    ntt_fwd_one(tmp, N, Q, rp);
    for (uint32_t i = 0; i < N; ++i) b[i] = addmod(orc_mulmod(a[i], s_ntt[i], Q), tmp[i], Q);
}

int orc_cbs_keygen(const orc_cbs_params *p, double sigma_lwe, double sigma_rlwe, uint32_t qks, uint32_t base_ks,
                   uint64_t seed, int32_t *s_lwe_out, int32_t *s_rlwe_out, uint64_t *bsk_out, uint64_t *ht_out,
                   uint64_t *ss_out, uint16_t *ksk_out, uint64_t *tv_out, uint64_t *gpow_out, uint32_t *maps_out) {
    const uint32_t N = p->N, n = p->n, log_n = p->log_n, l2 = 2 * p->digits_g, rounds = p->trace_rounds;
    const uint64_t Q = p->Q;
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * N), *irp = (uint64_t *)malloc(sizeof(uint64_t) * N);
    uint64_t ninv[2];
    if (orc_ntt_tables(log_n, Q, rp, NULL, irp, NULL, ninv) != 0) {
        free(rp);
        free(irp);
        return -1;
    }
    orc_rng r;
    rng_seed(&r, seed);
    int32_t *s_lwe = (int32_t *)malloc(sizeof(int32_t) * n), *s_rlwe = (int32_t *)malloc(sizeof(int32_t) * N);
    uint64_t *s_ntt = (uint64_t *)malloc(sizeof(uint64_t) * N), *tmp = (uint64_t *)malloc(sizeof(uint64_t) * N);
    uint64_t *a_scr = (uint64_t *)malloc(sizeof(uint64_t) * 2 * N);
    for (uint32_t i = 0; i < n; ++i) s_lwe[i] = (int32_t)(rng_next(&r) & 1);
    for (uint32_t i = 0; i < N; ++i) s_rlwe[i] = (int32_t)rng_uniform(&r, 3) - 1;
    for (uint32_t i = 0; i < N; ++i) s_ntt[i] = mod_signed(s_rlwe[i], Q);
    ntt_fwd_one(s_ntt, N, Q, rp);

    /* BSK: rows r = 2j + poly carry s_i g_j on component poly */
    uint64_t gbr[64], ght[64], gss[64];
    gadget_powers(Q, p->base_g, p->digits_g, gbr);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t row = 0; row < l2; ++row) {
            uint64_t *a = bsk_out ? bsk_out + ((size_t)i * l2 + row) * 2 * N : a_scr;
            uint64_t *b = a + N;
            keygen_rlwe_zero(&r, N, Q, sigma_rlwe, rp, s_ntt, a, b, tmp);
            if (s_lwe[i]) {
                uint64_t *tgt = (row & 1) ? b : a;
                for (uint32_t c = 0; c < N; ++c) tgt[c] = addmod(tgt[c], gbr[row >> 1], Q);
            }
        }

    /* HomTrace keys: automorphism X -> X^(N/2^r + 1) of s */
    gadget_powers(Q, p->base_ht, p->digits_ht, ght);
    uint64_t *sig = (uint64_t *)malloc(sizeof(uint64_t) * N);
    for (uint32_t rd = 0; rd < rounds; ++rd) {
        const uint64_t kk = ((uint64_t)N >> rd) + 1;
        memset(sig, 0, sizeof(uint64_t) * N);
        for (uint32_t i = 0; i < N; ++i) {
            const uint64_t e = ((uint64_t)i * kk) % (2ull * N);
            if (e < N) sig[e] = addmod(sig[e], mod_signed(s_rlwe[i], Q), Q);
            else sig[e - N] = addmod(sig[e - N], mod_signed(-(int64_t)s_rlwe[i], Q), Q);
        }
        ntt_fwd_one(sig, N, Q, rp);
        for (uint32_t j = 0; j < p->digits_ht; ++j) {
            uint64_t *a = ht_out ? ht_out + ((size_t)rd * p->digits_ht + j) * 2 * N : a_scr;
            uint64_t *b = a + N;
            keygen_rlwe_zero(&r, N, Q, sigma_rlwe, rp, s_ntt, a, b, tmp);
            for (uint32_t c = 0; c < N; ++c) b[c] = submod(b[c], orc_mulmod(sig[c], ght[j], Q), Q);
        }
    }
    free(sig);

    /* SchemeSwitch key: s^2 g_j */
    gadget_powers(Q, p->base_ss, p->digits_ss, gss);
    for (uint32_t j = 0; j < p->digits_ss; ++j) {
        uint64_t *a = ss_out ? ss_out + (size_t)j * 2 * N : a_scr;
        uint64_t *b = a + N;
        keygen_rlwe_zero(&r, N, Q, sigma_rlwe, rp, s_ntt, a, b, tmp);
        for (uint32_t c = 0; c < N; ++c)
            b[c] = addmod(b[c], orc_mulmod(orc_mulmod(s_ntt[c], s_ntt[c], Q), gss[j], Q), Q);
    }

    /* derived tables: gadget powers of the RGSW output, the multi-value test vector (slot j of
     * every 2^bw block holds -+g_j/2, negative on the first half), the automorphism maps */
    uint64_t gcc[64];
    gadget_powers(Q, p->base_cc, p->num_lut, gcc);
    if (gpow_out) memcpy(gpow_out, gcc, sizeof(uint64_t) * p->num_lut);
    if (tv_out) {
        uint32_t bw = 0;
        while ((1u << bw) < p->num_lut) ++bw;
        for (uint32_t i = 0; i < N; ++i) {
            const uint32_t slot = i & ((1u << bw) - 1);
            tv_out[i] = 0;
            if (slot >= p->num_lut) continue;
            const uint64_t half = (gcc[slot] >> 1) % Q;
            tv_out[i] = (i < N / 2) ? (half ? Q - half : 0) : half;
        }
    }
    if (maps_out) orc_auto_maps(maps_out, N, rounds);

    /* extraction key switch N -> n: LWE_s(v s'_i B^j) mod qks, u16 */
    const uint32_t outlen = n + 1, mask = qks - 1;
    uint16_t *row_scr = (uint16_t *)malloc(sizeof(uint16_t) * outlen);
    for (uint32_t j = 0; j < 2; ++j) {
        const uint32_t bj = (j == 0) ? 1u : base_ks;
        for (uint32_t i = 0; i < N; ++i) {
            const uint32_t si = (uint32_t)(s_rlwe[i] + (int32_t)qks) & mask;
            for (uint32_t v = 0; v < base_ks; ++v) {
                uint16_t *row = ksk_out ? ksk_out + (((size_t)j * N + i) * base_ks + v) * outlen : row_scr;
                uint32_t acc = 0;
                for (uint32_t c = 0; c < n; ++c) {
                    const uint32_t a = (uint32_t)(rng_next(&r) & mask);
                    row[c] = (uint16_t)a;
                    if (s_lwe[c]) acc += a;
                }
                const int64_t e = rng_rounded_gaussian(&r, sigma_lwe);
                const uint32_t m = (v * si * bj) & mask;
                row[n] = (uint16_t)((acc + m + (uint32_t)e) & mask);
            }
        }
    }
    free(row_scr);
    if (s_lwe_out) memcpy(s_lwe_out, s_lwe, sizeof(int32_t) * n);
    if (s_rlwe_out) memcpy(s_rlwe_out, s_rlwe, sizeof(int32_t) * N);
    free(a_scr);
    free(tmp);
    free(s_ntt);
    free(s_rlwe);
    free(s_lwe);
    free(irp);
    free(rp);
    return 0;
}

void orc_cbs_keygen_mb(const orc_cbs_params *p, double sigma_rlwe, const int32_t *s_lwe, const int32_t *s_rlwe,
                       uint32_t mb, uint64_t seed, uint64_t *mbk) {
    const uint32_t N = p->N, n = p->n, l2 = 2 * p->digits_g, K = orc_mb_keys(mb), groups = (n + mb - 1) / mb;
    const uint64_t Q = p->Q;
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * N), *irp = (uint64_t *)malloc(sizeof(uint64_t) * N);
    uint64_t ninv[2];
    orc_ntt_tables(p->log_n, Q, rp, NULL, irp, NULL, ninv);
    uint64_t *s_ntt = (uint64_t *)malloc(sizeof(uint64_t) * N);
    for (uint32_t i = 0; i < N; ++i) s_ntt[i] = mod_signed(s_rlwe[i], Q);
    ntt_fwd_one(s_ntt, N, Q, rp);
    uint64_t gbr[64];
    gadget_powers(Q, p->base_g, p->digits_g, gbr);
#pragma omp parallel for schedule(dynamic)
    for (long g = 0; g < (long)groups; ++g) {
        uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * N);
        orc_rng r;
        rng_seed(&r, seed ^ (0x9e3779b97f4a7c15ull * (uint64_t)(g + 1)));
        for (uint32_t kk = 0; kk < K; ++kk) {
            const uint32_t mask = orc_mb_mask(mb, kk);
            uint32_t prod = 1;
            for (uint32_t i = 0; i < mb; ++i)
                if (mask & (1u << i)) {
                    const uint32_t idx = (uint32_t)g * mb + i;
                    prod &= idx < n ? (uint32_t)s_lwe[idx] : 0u;
                }
            for (uint32_t row = 0; row < l2; ++row) {
                uint64_t *a = mbk + (((size_t)g * K + kk) * l2 + row) * 2 * N;
                uint64_t *b = a + N;
                keygen_rlwe_zero(&r, N, Q, sigma_rlwe, rp, s_ntt, a, b, tmp);
                if (prod) {
                    uint64_t *tgt = (row & 1) ? b : a;
                    for (uint32_t c = 0; c < N; ++c) tgt[c] = addmod(tgt[c], gbr[row >> 1], Q);
                }
            }
        }
        free(tmp);
    }
    free(s_ntt);
    free(irp);
    free(rp);
}

/* ------------------------------------------------------------------------------------------ */
/* key generation on the device, restated (ChaCha20-addressed words)                           */
/* ------------------------------------------------------------------------------------------ */

/* RLWE(0) sample (sample, domain): a = NTT-domain mask, b = a s + NTT(e) */
static void chacha_rlwe_zero(const uint32_t key[8], uint32_t sample, uint32_t domain, uint32_t N, uint64_t Q,
                             const uint64_t *rp, const uint64_t *s_ntt, const uint64_t *T, uint32_t tlen, uint64_t *a,
                             uint64_t *b, uint64_t *tmp) {
    const uint32_t nonce[3] = {sample, domain, 0u};
    for (uint32_t i = 0; i < N; ++i) {
        uint32_t blk[16];
        orc_chacha20_block(key, i, nonce, blk);
        a[i] = orc_uniform_mod(blk, Q);
        const int64_t e = orc_cdt_sample((uint64_t)blk[4] | ((uint64_t)blk[5] << 32), T, tlen);
        tmp[i] = e < 0 ? Q - (uint64_t)(-e) : (uint64_t)e;
    }
    ntt_fwd_one(tmp, N, Q, rp);
    for (uint32_t i = 0; i < N; ++i) b[i] = addmod(orc_mulmod(a[i], s_ntt[i], Q), tmp[i], Q);
}

static void chacha_secrets(const uint32_t key[8], uint32_t n, uint32_t N, int32_t *s_lwe, int32_t *s_rlwe) {
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t blk[16];
        const uint32_t nonce[3] = {0u, 3u, 0u};
        orc_chacha20_block(key, i, nonce, blk);
        s_lwe[i] = (int32_t)(blk[0] & 1u);
    }
    for (uint32_t i = 0; i < N; ++i) {
        uint32_t blk[16];
        const uint32_t nonce[3] = {1u, 3u, 0u};
        orc_chacha20_block(key, i, nonce, blk);
        s_rlwe[i] = (int32_t)orc_uniform_mod(blk, 3) - 1;
    }
}

int orc_cbs_keygen_chacha(const orc_cbs_params *p, double sigma_lwe, double sigma_rlwe, uint32_t qks,
                          uint32_t base_ks, const uint32_t key[8], int32_t *s_lwe_out, int32_t *s_rlwe_out,
                          uint64_t *bsk_out, uint64_t *ht_out, uint64_t *ss_out, uint16_t *ksk_out) {
    const uint32_t N = p->N, n = p->n, l2 = 2 * p->digits_g, rounds = p->trace_rounds;
    const uint64_t Q = p->Q;
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * N), *irp = (uint64_t *)malloc(sizeof(uint64_t) * N);
    uint64_t ninv[2];
    if (orc_ntt_tables(p->log_n, Q, rp, NULL, irp, NULL, ninv) != 0) {
        free(rp);
        free(irp);
        return -1;
    }
    uint64_t TR[4096], TL[4096];
    const uint32_t lr = orc_cdt_table(sigma_rlwe, TR, 4096), ll = orc_cdt_table(sigma_lwe, TL, 4096);
    int32_t *s_lwe = (int32_t *)malloc(sizeof(int32_t) * n), *s_rlwe = (int32_t *)malloc(sizeof(int32_t) * N);
    chacha_secrets(key, n, N, s_lwe, s_rlwe);
    uint64_t *s_ntt = (uint64_t *)malloc(sizeof(uint64_t) * N);
    for (uint32_t i = 0; i < N; ++i) s_ntt[i] = s_rlwe[i] < 0 ? Q - 1 : (uint64_t)s_rlwe[i];
    ntt_fwd_one(s_ntt, N, Q, rp);
    uint64_t gbr[64], ght[64], gss[64];
    gadget_powers(Q, p->base_g, p->digits_g, gbr);
    gadget_powers(Q, p->base_ht, p->digits_ht, ght);
    gadget_powers(Q, p->base_ss, p->digits_ss, gss);

    if (bsk_out) {
#pragma omp parallel for schedule(dynamic)
        for (long smp = 0; smp < (long)n * l2; ++smp) {
            uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * N);
            const uint32_t i = (uint32_t)(smp / l2), row = (uint32_t)(smp % l2);
            uint64_t *a = bsk_out + (size_t)smp * 2 * N, *b = a + N;
            chacha_rlwe_zero(key, (uint32_t)smp, 4u, N, Q, rp, s_ntt, TR, lr, a, b, tmp);
            if (s_lwe[i]) {
                uint64_t *tgt = (row & 1) ? b : a;
                for (uint32_t c = 0; c < N; ++c) tgt[c] = addmod(tgt[c], gbr[row >> 1], Q);
            }
            free(tmp);
        }
    }
    if (ht_out) {
        uint64_t *sig = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)rounds * N);
        for (uint32_t rd = 0; rd < rounds; ++rd) {
            const uint64_t kk = ((uint64_t)N >> rd) + 1;
            uint64_t *sg = sig + (size_t)rd * N;
            for (uint32_t i = 0; i < N; ++i) {
                const uint64_t e = ((uint64_t)i * kk) % (2ull * N);
                const int32_t v = e < N ? s_rlwe[i] : -s_rlwe[i];
                sg[e % N] = v < 0 ? Q - (uint64_t)(-v) : (uint64_t)v;
            }
            ntt_fwd_one(sg, N, Q, rp);
        }
#pragma omp parallel for schedule(dynamic)
        for (long smp = 0; smp < (long)rounds * p->digits_ht; ++smp) {
            uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * N);
            const uint32_t rd = (uint32_t)(smp / p->digits_ht), j = (uint32_t)(smp % p->digits_ht);
            uint64_t *a = ht_out + (size_t)smp * 2 * N, *b = a + N;
            chacha_rlwe_zero(key, (uint32_t)smp, 5u, N, Q, rp, s_ntt, TR, lr, a, b, tmp);
            for (uint32_t c = 0; c < N; ++c) b[c] = submod(b[c], orc_mulmod(sig[(size_t)rd * N + c], ght[j], Q), Q);
            free(tmp);
        }
        free(sig);
    }
    if (ss_out) {
        uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * N);
        for (uint32_t j = 0; j < p->digits_ss; ++j) {
            uint64_t *a = ss_out + (size_t)j * 2 * N, *b = a + N;
            chacha_rlwe_zero(key, j, 6u, N, Q, rp, s_ntt, TR, lr, a, b, tmp);
            for (uint32_t c = 0; c < N; ++c)
                b[c] = addmod(b[c], orc_mulmod(orc_mulmod(s_ntt[c], s_ntt[c], Q), gss[j], Q), Q);
        }
        free(tmp);
    }
    if (ksk_out) {
        const uint32_t mask = qks - 1, outlen = n + 1;
#pragma omp parallel for schedule(static)
        for (long t = 0; t < (long)2 * N * base_ks; ++t) {
            const uint32_t v = (uint32_t)(t % base_ks), i = (uint32_t)((t / base_ks) % N), j = (uint32_t)(t / ((long)base_ks * N));
            uint16_t *row = ksk_out + (size_t)t * outlen;
            const uint32_t nonce[3] = {(uint32_t)t, 7u, 0u};
            uint32_t acc = 0, blk[16];
            for (uint32_t c = 0; c < n; ++c) {
                orc_chacha20_block(key, c, nonce, blk);
                const uint32_t a = (uint32_t)orc_uniform_mod(blk, qks);
                row[c] = (uint16_t)a;
                if (s_lwe[c]) acc += a;
            }
            orc_chacha20_block(key, n, nonce, blk);
            const int64_t e = orc_cdt_sample((uint64_t)blk[4] | ((uint64_t)blk[5] << 32), TL, ll);
            const uint32_t si = (uint32_t)(s_rlwe[i] + (int32_t)qks) & mask;
            const uint32_t bj = j == 0 ? 1u : base_ks;
            const uint32_t m = (v * si * bj) & mask;
            row[n] = (uint16_t)((acc + m + (uint32_t)(int32_t)e) & mask);
        }
    }
    if (s_lwe_out) memcpy(s_lwe_out, s_lwe, sizeof(int32_t) * n);
    if (s_rlwe_out) memcpy(s_rlwe_out, s_rlwe, sizeof(int32_t) * N);
    free(s_ntt);
    free(s_rlwe);
    free(s_lwe);
    free(irp);
    free(rp);
    return 0;
}

void orc_cbs_keygen_chacha_mb(const orc_cbs_params *p, double sigma_rlwe, const uint32_t key[8],
                              const int32_t *s_lwe, const int32_t *s_rlwe, uint32_t mb, uint64_t *mbk) {
    const uint32_t N = p->N, n = p->n, l2 = 2 * p->digits_g, K = orc_mb_keys(mb), groups = (n + mb - 1) / mb;
    const uint64_t Q = p->Q;
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * N), *irp = (uint64_t *)malloc(sizeof(uint64_t) * N);
    uint64_t ninv[2];
    orc_ntt_tables(p->log_n, Q, rp, NULL, irp, NULL, ninv);
    uint64_t TR[4096];
    const uint32_t lr = orc_cdt_table(sigma_rlwe, TR, 4096);
    uint64_t *s_ntt = (uint64_t *)malloc(sizeof(uint64_t) * N);
    for (uint32_t i = 0; i < N; ++i) s_ntt[i] = s_rlwe[i] < 0 ? Q - 1 : (uint64_t)s_rlwe[i];
    ntt_fwd_one(s_ntt, N, Q, rp);
    uint64_t gbr[64];
    gadget_powers(Q, p->base_g, p->digits_g, gbr);
#pragma omp parallel for schedule(dynamic)
    for (long smp = 0; smp < (long)groups * K * l2; ++smp) {
        uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * N);
        const uint32_t row = (uint32_t)(smp % l2), kk = (uint32_t)((smp / l2) % K), g = (uint32_t)(smp / ((long)l2 * K));
        const uint32_t mask = orc_mb_mask(mb, kk);
        uint32_t prod = 1;
        for (uint32_t i = 0; i < mb; ++i)
            if (mask & (1u << i)) {
                const uint32_t idx = g * mb + i;
                prod &= idx < n ? (uint32_t)s_lwe[idx] : 0u;
            }
        uint64_t *a = mbk + (size_t)smp * 2 * N, *b = a + N;
        chacha_rlwe_zero(key, (uint32_t)smp, mb == 2 ? 8u : (mb == 3 ? 9u : 10u), N, Q, rp, s_ntt, TR, lr, a, b, tmp);
        if (prod) {
            uint64_t *tgt = (row & 1) ? b : a;
            for (uint32_t c = 0; c < N; ++c) tgt[c] = addmod(tgt[c], gbr[row >> 1], Q);
        }
        free(tmp);
    }
    free(s_ntt);
    free(irp);
    free(rp);
}

/* ------------------------------------------------------------------------------------------ */
/* LMKCDEY blind rotation (bitwise/src/cirbts/cirbts-lmkcdey.cu, keys cirbts-init.cu:630-726)   */
/* ------------------------------------------------------------------------------------------ */

static uint64_t lmk_pow5(uint32_t k, uint32_t M) {
    uint64_t v = 1;
    for (uint32_t i = 0; i < k; ++i) v = (v * 5) % M;
    return v;
}

/* automorphism powers of the key set (cirbts-lmkcdey.cu:66-103): pows[0] = 2N - 5, then
 * 5^i mod 2N for i = 1 .. num_auto_keys (window <= 1), or for window > 1 the powers 5^1 .. 5^window
 * followed by 5^(2 window), 5^(3 window), ... up to N/2 - 1 (5^window is not repeated);
 * returns the count.  pows may be NULL (count only). */
uint32_t orc_lmkcdey_auto_pows(uint32_t N, uint32_t num_auto_keys, uint32_t window, uint32_t *pows) {
    const uint32_t M = 2 * N, Nh = N / 2;
    uint32_t c = 0;
    if (pows) pows[c] = M - 5;
    ++c;
    if (window > 1) {
        for (uint32_t k = 1; k <= window; ++k) {
            if (pows) pows[c] = (uint32_t)lmk_pow5(k, M);
            ++c;
        }
        for (uint32_t k = 2 * window; k <= Nh - 1; k += window) {
            if (pows) pows[c] = (uint32_t)lmk_pow5(k, M);
            ++c;
        }
    } else {
        for (uint32_t k = 1; k <= num_auto_keys; ++k) {
            if (pows) pows[c] = (uint32_t)lmk_pow5(k, M);
            ++c;
        }
    }
    return c;
}

/* NTT-domain permutation of X -> X^k for every power: slot t holds the evaluation at
 * zeta^(2 brev(t) + 1), so psi_k(p) at slot t is p at the slot of zeta^((2 brev(t) + 1) k);
 * maps [count][N], out[t] = in[map[t]] as kernel_Permute_Only reads it (kernel.cu:7588) */
void orc_lmkcdey_auto_maps(uint32_t N, uint32_t num_auto_keys, uint32_t window, uint32_t *maps) {
    uint32_t log_n = 0;
    while ((1u << log_n) < N) ++log_n;
    const uint32_t count = orc_lmkcdey_auto_pows(N, num_auto_keys, window, NULL);
    uint32_t *pows = (uint32_t *)malloc(sizeof(uint32_t) * count);
    orc_lmkcdey_auto_pows(N, num_auto_keys, window, pows);
    for (uint32_t k = 0; k < count; ++k)
        for (uint32_t t = 0; t < N; ++t) {
            const uint64_t e = 2ull * brev(t, log_n) + 1;
            const uint32_t idx = (uint32_t)(((e * pows[k]) & (2ull * N - 1)) >> 1);
            maps[(size_t)k * N + t] = brev(idx, log_n);
        }
    free(pows);
}

/* approximate signed digit idx of x (kernel.cu:887-915): the centred value split into signed
 * g-bit digits from the least significant end, the first digit dropped */
static uint64_t lmk_digit(uint64_t x, uint64_t Q, int g, uint32_t idx) {
    int64_t d = x < (Q >> 1) ? (int64_t)x : (int64_t)x - (int64_t)Q;
    int64_t r = (int64_t)((uint64_t)d << (64 - g)) >> (64 - g);
    d = (d - r) >> g;
    for (uint32_t k = 0; k <= idx; ++k) {
        r = (int64_t)((uint64_t)d << (64 - g)) >> (64 - g);
        d = (d - r) >> g;
    }
    return r < 0 ? (uint64_t)(r + (int64_t)Q) : (uint64_t)r;
}

/* LMKCDEY keys from the secrets: eval [n][2 digits_g][2][N] = RGSW(X^{s_i}) with gadget
 * powers 2^{g (j + 1)} (row 2j carries the message on component a, row 2j + 1 on b);
 * autok [count][digits_g][2][N] = RLWE(0) with b -= 2^{g (j + 1)} psi_k(s) for every power k
 * of orc_lmkcdey_auto_pows.  One generator per key: eval key i seeded with
 * seed ^ (0x9e3779b97f4a7c15 (i + 1)), automorphism key k with
 * seed ^ 0x6c6d6b6364657921 ^ (0x9e3779b97f4a7c15 (k + 1)). */
void orc_lmkcdey_keygen(const orc_cbs_params *p, double sigma_rlwe, const int32_t *s_lwe, const int32_t *s_rlwe,
                        uint32_t num_auto_keys, uint32_t window, uint64_t seed, uint64_t *eval, uint64_t *autok) {
    const uint32_t N = p->N, n = p->n, dg = p->digits_g, M = 2 * N;
    const int g = __builtin_ctz(p->base_g);
    const uint64_t Q = p->Q;
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * N), *irp = (uint64_t *)malloc(sizeof(uint64_t) * N);
    uint64_t ninv[2];
    orc_ntt_tables(p->log_n, Q, rp, NULL, irp, NULL, ninv);
    uint64_t *s_ntt = (uint64_t *)malloc(sizeof(uint64_t) * N);
    for (uint32_t i = 0; i < N; ++i) s_ntt[i] = mod_signed(s_rlwe[i], Q);
    ntt_fwd_one(s_ntt, N, Q, rp);
    uint64_t gp[64];
    for (uint32_t j = 0; j < dg; ++j) {
        uint64_t v = 1 % Q;
        for (int e = 0; e < g * (int)(j + 1); ++e) v = addmod(v, v, Q);
        gp[j] = v;
    }
#pragma omp parallel for schedule(dynamic)
    for (long i = 0; i < (long)n; ++i) {
        uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * N), *mono = (uint64_t *)malloc(sizeof(uint64_t) * N);
        orc_rng r;
        rng_seed(&r, seed ^ (0x9e3779b97f4a7c15ull * (uint64_t)(i + 1)));
        const uint32_t e = (uint32_t)(((int64_t)s_lwe[i] % (int64_t)M + (int64_t)M) % (int64_t)M);
        memset(mono, 0, sizeof(uint64_t) * N);
        if (e < N) mono[e] = 1 % Q;
        else mono[e - N] = Q - 1;
        ntt_fwd_one(mono, N, Q, rp);
        for (uint32_t row = 0; row < 2 * dg; ++row) {
            uint64_t *a = eval + ((size_t)i * 2 * dg + row) * 2 * N, *b = a + N;
            keygen_rlwe_zero(&r, N, Q, sigma_rlwe, rp, s_ntt, a, b, tmp);
            uint64_t *tgt = (row & 1) ? b : a;
            for (uint32_t c = 0; c < N; ++c) tgt[c] = addmod(tgt[c], orc_mulmod(mono[c], gp[row >> 1], Q), Q);
        }
        free(mono);
        free(tmp);
    }
    const uint32_t count = orc_lmkcdey_auto_pows(N, num_auto_keys, window, NULL);
    uint32_t *maps = (uint32_t *)malloc(sizeof(uint32_t) * count * N);
    orc_lmkcdey_auto_maps(N, num_auto_keys, window, maps);
#pragma omp parallel for schedule(dynamic)
    for (long k = 0; k < (long)count; ++k) {
        uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * N);
        orc_rng r;
        rng_seed(&r, seed ^ 0x6c6d6b6364657921ull ^ (0x9e3779b97f4a7c15ull * (uint64_t)(k + 1)));
        const uint32_t *map = maps + (size_t)k * N;
        for (uint32_t j = 0; j < dg; ++j) {
            uint64_t *a = autok + ((size_t)k * dg + j) * 2 * N, *b = a + N;
            keygen_rlwe_zero(&r, N, Q, sigma_rlwe, rp, s_ntt, a, b, tmp);
            for (uint32_t c = 0; c < N; ++c) b[c] = submod(b[c], orc_mulmod(s_ntt[map[c]], gp[j], Q), Q);
        }
        free(tmp);
    }
    free(maps);
    free(s_ntt);
    free(irp);
    free(rp);
}

/* discrete log of odd x in Z_2N to base 5 with sign: w for x = 5^w, -w for x = -5^w (w >= 1),
 * 2N for x = -1 (the reference's logGen, cirbts-lmkcdey.cu:143-176) */
static void lmk_log_table(uint32_t N, int32_t *log_tab /* [N], index x >> 1 */) {
    const uint32_t M = 2 * N, Nh = N / 2;
    uint64_t v = 1;
    for (uint32_t w = 0; w < Nh; ++w) {
        log_tab[v >> 1] = (int32_t)w;
        const uint32_t neg = (uint32_t)(M - v);
        log_tab[neg >> 1] = w == 0 ? (int32_t)M : -(int32_t)w;
        v = (v * 5) % M;
    }
}

typedef struct {
    const orc_cbs_params *p;
    const uint64_t *eval, *autok;
    const uint32_t *maps;
    uint64_t *ct, *dct, *perm0, *perm1, *tmp;
    const uint64_t *rp, *irp;
    uint64_t n_inv;
} lmk_ctx;

/* AddToAccLMKCDEY_GPU (cirbts-lmkcdey.cu:239-259): acc <- acc (x) RGSW(X^{s_j}) */
static void lmk_add(lmk_ctx *c, uint64_t *acc, uint32_t j) {
    const orc_cbs_params *p = c->p;
    const uint32_t N = p->N, dg = p->digits_g;
    const int g = __builtin_ctz(p->base_g);
    const uint64_t Q = p->Q;
    const uint64_t *key = c->eval + (size_t)j * 2 * dg * 2 * N;
    memcpy(c->ct, acc, sizeof(uint64_t) * 2 * N);
    ntt_inv_one(c->ct, N, Q, c->irp, c->n_inv);
    ntt_inv_one(c->ct + N, N, Q, c->irp, c->n_inv);
    for (uint32_t d = 0; d < dg; ++d)
        for (uint32_t poly = 0; poly < 2; ++poly) {
            uint64_t *row = c->dct + (size_t)(2 * d + poly) * N;
            for (uint32_t i = 0; i < N; ++i) row[i] = lmk_digit(c->ct[poly * N + i], Q, g, d);
            ntt_fwd_one(row, N, Q, c->rp);
        }
    for (uint32_t i = 0; i < N; ++i) {
        uint64_t s0 = 0, s1 = 0;
        for (uint32_t r = 0; r < 2 * dg; ++r) {
            const uint64_t x = c->dct[(size_t)r * N + i];
            s0 = addmod(s0, orc_mulmod(x, key[(size_t)r * 2 * N + i], Q), Q);
            s1 = addmod(s1, orc_mulmod(x, key[(size_t)r * 2 * N + N + i], Q), Q);
        }
        acc[i] = s0;
        acc[N + i] = s1;
    }
}

/* AutomorphismLMKCDEY_GPU (cirbts-lmkcdey.cu:261-292): acc <- key switch of psi_k(acc) */
static void lmk_auto(lmk_ctx *c, uint64_t *acc, uint32_t k) {
    const orc_cbs_params *p = c->p;
    const uint32_t N = p->N, dg = p->digits_g;
    const int g = __builtin_ctz(p->base_g);
    const uint64_t Q = p->Q;
    const uint32_t *map = c->maps + (size_t)k * N;
    const uint64_t *key = c->autok + (size_t)k * dg * 2 * N;
    for (uint32_t i = 0; i < N; ++i) {
        c->perm1[i] = acc[N + map[i]];
        c->perm0[i] = acc[map[i]];
    }
    ntt_inv_one(c->perm0, N, Q, c->irp, c->n_inv);
    for (uint32_t d = 0; d < dg; ++d) {
        uint64_t *row = c->dct + (size_t)d * N;
        for (uint32_t i = 0; i < N; ++i) row[i] = lmk_digit(c->perm0[i], Q, g, d);
        ntt_fwd_one(row, N, Q, c->rp);
    }
    for (uint32_t i = 0; i < N; ++i) {
        uint64_t s0 = 0, s1 = 0;
        for (uint32_t d = 0; d < dg; ++d) {
            const uint64_t x = c->dct[(size_t)d * N + i];
            s0 = addmod(s0, orc_mulmod(x, key[(size_t)d * 2 * N + i], Q), Q);
            s1 = addmod(s1, orc_mulmod(x, key[(size_t)d * 2 * N + N + i], Q), Q);
        }
        acc[i] = s0;
        acc[N + i] = addmod(c->perm1[i], s1, Q);
    }
}

/* LMKCDEY_EvalAcc (cirbts-lmkcdey.cu:105-407, window 0) on acc [2][N] (NTT domain, in place):
 * a_neg [n] the masks mod 2N as the reference's EvalAcc receives them (negated by the caller,
 * cirbts-bootstrap.cu:681-689).  The LWE coefficients are bucketed by the signed base-5
 * logarithm of the odd residue (-a_neg) | 1, then processed bucket by bucket with
 * automorphisms between them. */
/* key index of the power 5^k in the key set of orc_lmkcdey_auto_pows */
static uint32_t lmk_key_index(uint32_t k, uint32_t window) {
    return (window > 1 && k > window) ? window + k / window - 1 : k;
}

/* the automorphisms closing a run of `skips` steps: 5^skips (non-windowed), or 5^(q window)
 * then 5^r for skips = q window + r (apply_skip, cirbts-lmkcdey.cu:311-325) */
static void lmk_skip(lmk_ctx *c, uint64_t *acc, uint32_t skips, uint32_t window) {
    if (window <= 1) {
        lmk_auto(c, acc, skips);
        return;
    }
    const uint32_t q = skips / window, r = skips % window;
    if (q) lmk_auto(c, acc, lmk_key_index(q * window, window));
    if (r) lmk_auto(c, acc, lmk_key_index(r, window));
}

void orc_lmkcdey_eval_acc(const orc_cbs_params *p, const uint64_t *eval, const uint64_t *autok, const uint32_t *maps,
                          uint32_t num_auto_keys, uint32_t window, const uint32_t *a_neg, uint32_t n, uint64_t *acc) {
    const uint32_t N = p->N, Nh = N / 2, M = 2 * N, mask = M - 1, buckets = 2 * Nh, dg = p->digits_g;
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * N), *irp = (uint64_t *)malloc(sizeof(uint64_t) * N);
    uint64_t ninv[2];
    orc_ntt_tables(p->log_n, p->Q, rp, NULL, irp, NULL, ninv);
    int32_t *log_tab = (int32_t *)malloc(sizeof(int32_t) * N);
    lmk_log_table(N, log_tab);
    uint32_t *bucket = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *offs = (uint32_t *)calloc(buckets + 1, sizeof(uint32_t));
    uint32_t *cur = (uint32_t *)malloc(sizeof(uint32_t) * (buckets + 1));
    uint32_t *items = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t odd = ((0u - a_neg[i]) & mask) | 1u;
        const int32_t idx = log_tab[odd >> 1];
        bucket[i] = idx == (int32_t)M ? buckets - 1 : (uint32_t)(idx + (int32_t)(Nh - 1));
        ++offs[bucket[i] + 1];
    }
    for (uint32_t b = 0; b < buckets; ++b) offs[b + 1] += offs[b];
    memcpy(cur, offs, sizeof(uint32_t) * (buckets + 1));
    for (uint32_t i = 0; i < n; ++i) items[cur[bucket[i]]++] = i;

    lmk_ctx c;
    c.p = p;
    c.eval = eval;
    c.autok = autok;
    c.maps = maps;
    c.rp = rp;
    c.irp = irp;
    c.n_inv = ninv[0];
    c.ct = (uint64_t *)malloc(sizeof(uint64_t) * 2 * N);
    c.dct = (uint64_t *)malloc(sizeof(uint64_t) * 2 * dg * N);
    c.perm0 = (uint64_t *)malloc(sizeof(uint64_t) * N);
    c.perm1 = (uint64_t *)malloc(sizeof(uint64_t) * N);
    c.tmp = NULL;

    /* acc1 = psi_{2N-5}(acc1) without key switching (the mask is 0) */
    for (uint32_t i = 0; i < N; ++i) c.perm1[i] = acc[N + maps[i]];
    memcpy(acc + N, c.perm1, sizeof(uint64_t) * N);
    for (int half = 0; half < 2; ++half) {
        /* half 0: a = -5^i (buckets 0 .. Nh-2), half 1: a = 5^i (buckets 2Nh-2 .. Nh) */
        uint32_t skips = 0;
        for (uint32_t i = Nh - 1; i > 0; --i) {
            const uint32_t b = half == 0 ? (Nh - 1) - i : (Nh - 1) + i;
            if (offs[b] != offs[b + 1]) {
                if (skips != 0) {
                    lmk_skip(&c, acc, skips, window);
                    skips = 0;
                }
                for (uint32_t pos = offs[b]; pos < offs[b + 1]; ++pos) lmk_add(&c, acc, items[pos]);
            }
            ++skips;
            if ((window <= 1 && skips == num_auto_keys) || i == 1) {
                lmk_skip(&c, acc, skips, window);
                skips = 0;
            }
        }
        if (half == 0) {
            /* a = -1, then psi_{2N-5} */
            for (uint32_t pos = offs[buckets - 1]; pos < offs[buckets]; ++pos) lmk_add(&c, acc, items[pos]);
            lmk_auto(&c, acc, 0);
        } else {
            /* a = 1 */
            for (uint32_t pos = offs[Nh - 1]; pos < offs[Nh]; ++pos) lmk_add(&c, acc, items[pos]);
        }
    }
    free(c.ct);
    free(c.dct);
    free(c.perm0);
    free(c.perm1);
    free(items);
    free(cur);
    free(offs);
    free(bucket);
    free(log_tab);
    free(irp);
    free(rp);
}

/* the circuit-bootstrapping blind rotation with the LMKCDEY accumulator
 * (cirbts-bootstrap.cu:600-720 with method LMKCDEY): acc = (0, X^{-b~} TV) with the special
 * mod switch of b, the masks rounded to Z_2N (the reference passes them unswitched, which is
 * the same when q_lwe = 2N) and negated, LMKCDEY_EvalAcc (which rounds them to odd), then the
 * finalize of the GINX form.  acc_out [batch][2][N] NTT domain. */
void orc_blind_rotate_lmkcdey(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *eval,
                              const uint64_t *autok, const uint32_t *maps, uint32_t num_auto_keys, uint32_t window,
                              const uint64_t *a,
                              const uint64_t *b, uint32_t batch, uint32_t a_stride, uint64_t *acc_out, int finalize) {
    const uint32_t N = p->N, twoN = 2 * N;
    const uint64_t Q = p->Q;
    const uint32_t bw = (p->num_lut <= 1) ? 0 : (uint32_t)(32 - __builtin_clz(p->num_lut - 1));
#pragma omp parallel for schedule(dynamic, 1)
    for (long bi = 0; bi < (long)batch; ++bi) {
        uint64_t *acc = acc_out + (size_t)bi * 2 * N;
        const uint64_t *arow = a + (size_t)bi * a_stride;
        uint32_t *a_neg = (uint32_t *)malloc(sizeof(uint32_t) * (p->n ? p->n : 1));
        for (uint32_t i = 0; i < p->n; ++i) a_neg[i] = (twoN - orc_special_ms(arow[i], twoN, p->q_lwe, 0)) & (twoN - 1);
        const uint32_t bt = orc_special_ms(b[bi], twoN, p->q_lwe, bw);
        memset(acc, 0, sizeof(uint64_t) * N);
        rotate_neg(acc + N, k->tv, bt, N, Q);
        ntt_fwd_one(acc + N, N, Q, k->rp);
        orc_lmkcdey_eval_acc(p, eval, autok, maps, num_auto_keys, window, a_neg, p->n, acc);
        free(a_neg);
        if (finalize) {
            const uint64_t ninv = orc_invmod(N, Q);
            for (uint32_t c = 0; c < 2 * N; ++c) acc[c] = orc_mulmod(acc[c], ninv, Q);
            ntt_inv_one(acc, N, Q, k->irp, k->n_inv);
            ntt_inv_one(acc + N, N, Q, k->irp, k->n_inv);
            for (uint32_t j = 0; j < p->num_lut; ++j)
                acc[N + j] = addmod(acc[N + j], orc_mulmod(k->gpow[j] >> 1, ninv, Q), Q);
            ntt_fwd_one(acc, N, Q, k->rp);
            ntt_fwd_one(acc + N, N, Q, k->rp);
        }
    }
}
