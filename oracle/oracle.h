/*
 * oracle.h -- CPU restatement of the reference's bootstrapping hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference
 * legs may load it.  The product library never links or calls it.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths relative to the reference project root).  All modular arithmetic is
 * exact (unsigned __int128); results are fully reduced to [0, q).
 *
 * Pinning: the Phantom NTT tables, get_primes and the plaintext AES are checked
 * against the reference's own host code compiled from its sources (oracle/_ref,
 * recipe in oracle/Makefile) and against committed golden fixtures generated from
 * it (tests/golden/make_golden.py), plus the FIPS-197 AES-128 known answer.
 * The CBS / CMux / extract restatements follow the cited kernels; the keys and
 * parameter sets they consume come from the OpenFHE fork, which is absent, so
 * those stages are "parity unpinned" against the reference and are pinned only
 * end to end (decrypted AES output == plaintext AES-128).
 */
#ifndef CBS_ORACLE_H
#define CBS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- scalar modular arithmetic (include/uintmodmath.cuh) ---------------- */
uint64_t orc_mulmod(uint64_t a, uint64_t b, uint64_t q);
uint64_t orc_powmod(uint64_t a, uint64_t e, uint64_t q);
uint64_t orc_invmod(uint64_t a, uint64_t q);
uint64_t orc_shoup(uint64_t w, uint64_t q);
int orc_is_prime(uint64_t n);
/* src/host/numth.cu:207-233 get_primes(ntt_size, bit_size, count) */
int orc_get_primes(uint32_t ntt_size, int bit_size, uint32_t count, uint64_t *out);
/* src/host/numth.cu:309-331 try_minimal_primitive_root */
uint64_t orc_minimal_primitive_root(uint64_t degree, uint64_t q);

/* ---------------- Phantom single-modulus NTT (src/host/ntt.cu:11-56, src/ntt/ntt_1d.cu) ---------------- */
/* rp/rp_sh/irp/irp_sh: N entries each; n_inv[0]=N^-1 mod q, n_inv[1]=its Shoup quotient */
int orc_ntt_tables(uint32_t log_n, uint64_t q, uint64_t *rp, uint64_t *rp_sh, uint64_t *irp, uint64_t *irp_sh,
                   uint64_t *n_inv);
/* ntt_1d.cu:488 inplace_fnwt_radix2_opt_batched: bit-reversed output, fully reduced */
void orc_ntt_forward(uint64_t *a, size_t batch, uint32_t n, uint64_t q, const uint64_t *rp);
/* ntt_1d.cu:557 inplace_inwt_radix2_batched (n^-1 fused) */
void orc_ntt_inverse(uint64_t *a, size_t batch, uint32_t n, uint64_t q, const uint64_t *irp, uint64_t n_inv);
/* ntt_1d.cu:677 inplace_inwt_radix2_permute_batched: in[map[i]] (negated when map>=n), then INTT */
void orc_ntt_inverse_permute(uint64_t *out, const uint64_t *in, const uint32_t *map, size_t batch, uint32_t n,
                             uint64_t q, const uint64_t *irp, uint64_t n_inv);
/* schoolbook negacyclic product c = a*b mod (X^n+1, q) (for checking the transform) */
void orc_negacyclic_mul(const uint64_t *a, const uint64_t *b, uint64_t *c, uint32_t n, uint64_t q);
/* bitwise/src/cirbts/kernel.cu:7554-7571 kernel_GenerateCoefficientAutoMaps (NTT-domain automorphism maps) */
void orc_auto_maps(uint32_t *maps, uint32_t n, uint32_t levels);

/* ---------------- gadget decomposition / mod switch ---------------- */
/* bitwise/src/cirbts/kernel.cu:37-68 device_SignedDigitDecompose2: digits in [0,Q) (negatives as Q-|r|) */
void orc_signed_decompose(uint64_t x, uint64_t Q, uint32_t base, uint32_t digits, uint64_t *out);
/* bitwise/src/cirbts/kernel.cu:7316-7326 device_SpecialMS_IndexPos */
uint32_t orc_special_ms(uint64_t v, uint32_t two_n, uint64_t q, uint32_t bitwidth);

/* ---------------- circuit bootstrapping (bitwise/src/cirbts) ---------------- */
typedef struct {
    uint32_t N;          /* ring dimension */
    uint32_t log_n;
    uint64_t Q;          /* RLWE modulus (NTT prime) */
    uint32_t n;          /* LWE dimension */
    uint64_t q_lwe;      /* LWE modulus of the CBS input */
    uint32_t base_g;     /* blind-rotation gadget base (power of two) */
    uint32_t digits_g;   /* blind-rotation gadget digits */
    uint32_t num_lut;    /* = digitsCC, RGSW levels produced */
    uint32_t base_cc;    /* CMux / RGSW output gadget base */
    uint32_t base_ht, digits_ht;
    uint32_t base_ss, digits_ss;
    uint32_t trace_rounds;
} orc_cbs_params;

typedef struct {
    const uint64_t *rp, *irp;   /* Phantom tables for (N, Q) */
    uint64_t n_inv;
    const uint32_t *auto_maps;  /* [log_n][N] */
    const uint64_t *tv;         /* blind-rotation test vector, coefficient domain [N] */
    const uint64_t *gpow;       /* [num_lut] RGSW gadget powers */
    const uint64_t *bsk;        /* [n][2*digits_g][2][N] NTT domain */
    const uint64_t *ht_key;     /* [trace_rounds][digits_ht][2][N] NTT domain */
    const uint64_t *ss_key;     /* [digits_ss][2][N] NTT domain */
} orc_cbs_keys;

/* cirbts-batch.cu:3293-4629 (binary GINX EvalAcc) + finalize :2622-2642.
 * acc_out [batch][2][N] NTT domain. */
void orc_blind_rotate(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *a, const uint64_t *b,
                      uint32_t batch, uint32_t a_stride, uint64_t *acc_out, int finalize);
/* Multi-bit blind rotation, mb = 2, 3 or 4 (cirbts-init.cu:376-565 key grouping,
 * kernel.cu:4585-4771, MB4 staging cirbts-batch.cu:2767-2923): mbk [ceil(n/mb)][keys][2*digits_g]
 * [2][N] NTT domain, keys = orc_mb_keys(mb), subsets in the order of orc_mb_mask: {0} {1} {2}
 * {0,1} {0,2} {1,2} {0,1,2} (mb = 3), {0} {1} {0,1} (mb = 2), {0} {1} {2} {3} {0,1} {0,2} {1,2}
 * {0,1,2} (mb = 4: the mb = 3 step of coefficients 0-2, then a one-bit step of coefficient 3). */
uint32_t orc_mb_keys(uint32_t mb);
uint32_t orc_mb_mask(uint32_t mb, uint32_t kk);
void orc_blind_rotate_mb(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *mbk, uint32_t mb,
                         const uint64_t *a, const uint64_t *b, uint32_t batch, uint32_t a_stride, uint64_t *acc_out,
                         int finalize);
/* BR + finalize + multi-value split (kernel.cu:7498-7536): mv [batch][num_lut][2][N] NTT domain */
void orc_blind_rotate_mv(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *a, const uint64_t *b,
                         uint32_t batch, uint32_t a_stride, uint64_t *mv);
/* cirbts-batch.cu:1416-1879 full CBS: BR -> MV split -> HomTrace -> SchemeSwitch.
 * rgsw_out [batch][num_lut][2][2][N] NTT domain, row (2j+0)=scheme-switch row, (2j+1)=trace row. */
void orc_circuit_bootstrap(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *a, const uint64_t *b,
                           uint32_t batch, uint32_t a_stride, uint64_t *rgsw_out);
/* HomTrace + SchemeSwitch alone on MV RLWEs ct [count][2][N] NTT domain -> rgsw [count][2][2][N] */
void orc_trace_schemeswitch(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *ct, uint32_t count,
                            uint64_t *rgsw_out);

/* ---------------- CMux LUT (examples/aes_transcipher/rlwe_tables.cuh:52-108, gpu_lut.cuh:521-595) ---------------- */
/* out = ct_in (x) rgsw, both NTT domain; rgsw [digits][2][2][N] */
void orc_external_product(const uint64_t *ct_in, const uint64_t *rgsw, uint64_t *out, uint32_t N, uint64_t Q,
                          const uint64_t *rp, const uint64_t *irp, uint64_t n_inv, uint32_t base, uint32_t digits);
/* table [256][2][N], ctrl[8] -> pointers to RGSW [digits][2][2][N] (bit 0 = LSB); out [2][N] */
void orc_lut8x32(const uint64_t *table, const uint64_t *const *ctrl, uint64_t *out, uint32_t N, uint64_t Q,
                 const uint64_t *rp, const uint64_t *irp, uint64_t n_inv, uint32_t base, uint32_t digits);

/* ---------------- sample extract + LWE key switch (examples/aes_gpu_ks.cuh:341-607) ---------------- */
/* words [W][2][N] coefficient domain (c0=a, c1=b); info[t] = (word<<16)|coeff; ksk [2][N][base][n+1] u16;
 * out_a [T][out_stride], out_b [T] mod q_lwe */
void orc_extract_keyswitch(const uint64_t *words_coef, const uint32_t *info, uint32_t T, uint32_t N, uint64_t Q,
                           const uint16_t *ksk, uint32_t n, uint32_t base_ks_log2, uint32_t qks, uint64_t q_lwe,
                           uint64_t *out_a, uint64_t *out_b, uint32_t out_stride);

/* ---------------- Phantom RNS NTT and hybrid key switching (CKKS path) ---------------- */
/* data [polys][limbs][2^log_n]; limb l uses prime q[l] with its Phantom tables
 * (src/ntt/fntt_2d.cu:620 nwt_2d_radix8_forward_inplace, intt_2d.cu:724 backward) */
void orc_rns_ntt(uint64_t *data, size_t polys, uint32_t limbs, uint32_t log_n, const uint64_t *q, int inverse);
/* src/rns_bconv.cu:530-634 DRNSTool::modup (CKKS): c2 [Ql][n] NTT -> out [beta][Ql+P][n] NTT,
 * alpha = size_p digits of Ql per beta */
void orc_modup(const uint64_t *c2, uint64_t *out, uint32_t log_n, const uint64_t *q, uint32_t size_ql,
               const uint64_t *p, uint32_t size_p);
/* src/eval_key_switch.cu:13-68: t [beta][Ql+P][n], evk [beta][2][Q+P][n] (key limbs: Q chain then P)
 * -> cx [2][Ql+P][n] */
void orc_ks_inner(const uint64_t *t, const uint64_t *evk, uint64_t *cx, uint32_t n, const uint64_t *q, uint32_t size_ql,
                  uint32_t size_q, const uint64_t *p, uint32_t size_p);
/* src/rns_bconv.cu:776-828 DRNSTool::moddown_from_NTT (CKKS): cx [Ql+P][n] NTT -> ct [Ql][n] NTT */
void orc_moddown(const uint64_t *cx, uint64_t *ct, uint32_t log_n, const uint64_t *q, uint32_t size_ql,
                 const uint64_t *p, uint32_t size_p);
/* src/eval_key_switch.cu:94-181 keyswitch_inplace (CKKS): ct [2][Ql][n] += moddown(inner(modup(c2))) */
void orc_keyswitch(uint64_t *ct, const uint64_t *c2, const uint64_t *evk, uint32_t log_n, const uint64_t *q,
                   uint32_t size_ql, uint32_t size_q, const uint64_t *p, uint32_t size_p);

/* ---------------- gate bootstrap on the 32-bit torus (TFHE form of binfhe's GINX) ---------------- */
typedef struct {
    uint32_t n, N, bg_bits, levels, ks_base_bits, ks_levels;
} orc_gate_params;
/* the linear part of a two-input gate (binfhe-base-scheme-batch.cu:82-110 in torus form):
 * gate 0 OR, 1 AND, 2 NOR, 3 NAND, 4 XOR, 5 XNOR; messages are +-1/8 */
void orc_gate_combine(int gate, const uint32_t *a1, uint32_t b1, const uint32_t *a2, uint32_t b2, uint32_t n,
                      uint32_t *a, uint32_t *b);
/* blind rotation with test vector 1/8 (binfhe-base-scheme-batch.cu:16-74, rgsw-acc-batch.cu):
 * bsk [n][2*levels][2][N] torus32 (row 2k+p: digit k of component p), exact integer products;
 * writes the extracted LWE of dimension N: ext[0..N-1] = a, ext[N] = b */
void orc_gate_blind_rotate(const orc_gate_params *p, const uint32_t *bsk, const uint32_t *a, uint32_t b,
                           uint32_t *ext);
/* the same with a constant test vector mu (instead of 1/8) and b_add added to the extracted b */
void orc_gate_blind_rotate_tv(const orc_gate_params *p, const uint32_t *bsk, const uint32_t *a, uint32_t b,
                              uint32_t mu, uint32_t b_add, uint32_t *ext);
/* level-2 blind rotation on the 64-bit torus (exact integer products mod 2^64), constant test
 * vector mu, b_add added to the extracted b: bsk [n][2*levels][2][N] u64, a/b level-0 torus32 */
void orc_tcb_blind_rotate64(const orc_gate_params *p, const uint64_t *bsk, const uint32_t *a, uint32_t b,
                            uint64_t mu, uint64_t b_add, uint64_t *ext);
/* Grouped (multi-bit, mb = 2 or 3) forms of the two torus blind rotations:
 * mbk [ceil(n/mb)][2^mb - 1][2*levels][2][N], subsets {0} {1} {2} {0,1} {0,2} {1,2} {0,1,2}
 * (mb = 3) or {0} {1} {0,1} (mb = 2). */
void orc_gate_blind_rotate_tv_mb(const orc_gate_params *p, const uint32_t *mbk, uint32_t mb, const uint32_t *a,
                                 uint32_t b, uint32_t mu, uint32_t b_add, uint32_t *ext);
void orc_tcb_blind_rotate64_mb(const orc_gate_params *p, const uint64_t *mbk, uint32_t mb, const uint32_t *a,
                               uint32_t b, uint64_t mu, uint64_t b_add, uint64_t *ext);
/* private functional key switch of an extracted torus64 LWE (a[N2], b) into a torus32 RLWE of
 * dimension N1 (CGGI 2017 Alg. 2): key [N2+1][levels][base-1][2][N1] = RLWE(f(v * y_i *
 * 2^(32-(j+1)*base_bits))), y_i = key_i (i < N2), y_N2 = 1; digits of the top 32 bits of
 * (-a, b) rounded */
void orc_tcb_pfks(uint32_t N2, uint32_t N1, uint32_t base_bits, uint32_t levels, const uint32_t *key,
                  const uint64_t *ext, uint32_t *out);
/* LWE key switch N -> n (binfhe-base-scheme-batch.cu:145-185): ksk [N][ks_levels][base-1][n+1] */
void orc_gate_keyswitch(const orc_gate_params *p, const uint32_t *ksk, const uint32_t *ext, uint32_t *out);
/* the rotation of an arbitrary test vector tv [N] (NULL: the constant mu) */
void orc_gate_blind_rotate_lut(const orc_gate_params *p, const uint32_t *bsk, const uint32_t *a, uint32_t b,
                               const uint32_t *tv, uint32_t mu, uint32_t b_add, uint32_t *ext);
/* the programmable bootstrap (binfhe-base-scheme-batch.cu:215-364): a [n], b mod 2^in_bits, lut
 * [2^in_bits / 2] values mod 2^f_bits; out [n + 1] mod 2^f_bits encrypting lut[phase] (negacyclic
 * above half) */
void orc_gate_bootstrap_func(const orc_gate_params *p, const uint32_t *bsk, const uint32_t *ksk, const uint32_t *a,
                             uint32_t b, uint32_t in_bits, const uint64_t *lut, uint32_t f_bits, uint32_t *out);

/* ---------------- plaintext AES-128 (examples/aes_transcipher/aes128.cuh) ---------------- */
void orc_aes128_key_expand(const uint8_t key[16], uint8_t round_keys[11][16]);
void orc_aes128_encrypt(const uint8_t key[16], const uint8_t in[16], uint8_t out[16]);
/* te[8][256]: Te0..Te3 then Te4_0..Te4_3 (aes128.cuh:316-330) */
void orc_aes_enc_tables(uint32_t te[8][256]);

/* OpenMP thread count used by the batched routines */
int orc_num_threads(void);

/* ---------------- encryption of the AES material (rlwe_tables.cuh:5-24,
 * key_material.cuh:12-46; the reference encrypts on the host through OpenFHE, whose
 * sampler is absent, so this restates the device design: ChaCha20 per coefficient,
 * floor(x q / 2^128) masks, discrete-Gaussian noise by cumulative table) ---------------- */

/* RFC 8439 s2.3 block function: state = constants, key[8], counter, nonce[3]; out[16] */
void orc_chacha20_block(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3], uint32_t out[16]);
/* floor(x q / 2^128), x = w[0] + w[1] 2^32 + w[2] 2^64 + w[3] 2^96 */
uint64_t orc_uniform_mod(const uint32_t w[4], uint64_t q);
/* T[k] = floor(2^63 P(|X| <= k)) of exp(-x^2 / 2 sigma^2) while below 2^63; returns the length */
uint32_t orc_cdt_table(double sigma, uint64_t *T, uint32_t cap);
/* sign = bit 63 of u, magnitude = #{k : (u mod 2^63) >= T[k]} */
int64_t orc_cdt_sample(uint64_t u, const uint64_t *T, uint32_t len);
/* RLWE (NTT domain) of count words, sample indices first.., bit j of a word -> floor(Q/2)
 * on coefficient j; out [count][2][N] */
void orc_encrypt_words_rlwe(const uint32_t key[8], const uint32_t *words, uint32_t count, uint32_t first, uint32_t N,
                            uint64_t Q, const uint64_t *rp, const uint64_t *s_ntt, const uint64_t *T, uint32_t tlen,
                            uint64_t *out);
/* LWE of count bits (floor(q/2) scaling) under the binary s[n]; a [count][n], b [count] */
void orc_encrypt_bits_lwe(const uint32_t key[8], const uint8_t *bits, uint32_t count, uint32_t n, uint64_t q,
                          const int32_t *s, const uint64_t *T, uint32_t tlen, uint64_t *a, uint64_t *b);

/* ---------------- key generation for the CPU legs (the reference generates its keys in the
 * absent OpenFHE fork: CirBTKeyGen / KeySwitchGen, examples/aes_transcipher/main.cu:232-252).
 * Restates the seeded host key generation of the CUDA path's host side, generator included
 * (xoshiro256** seeded through splitmix64, Box-Muller Gaussians rounded to integers), so the
 * same seed gives the same keys word for word: binary LWE secret, ternary RLWE secret, BSK
 * RGSW(s_i) [n][2 digits_g][2][N], HomTrace keys (k1 - k0 s = -sigma_r(s) g_j + e)
 * [rounds][digits_ht][2][N], SchemeSwitch key (k1 - k0 s = s^2 g_j + e) [digits_ss][2][N], all
 * NTT domain, the extraction KSK [2][N][base_ks][n+1] u16 mod qks, and the derived test vector
 * tv[N], gadget powers gpow[num_lut] and automorphism maps [rounds][N].  Any output may be
 * NULL.  Returns 0, or -1 for parameters without NTT tables. ---------------- */
int orc_cbs_keygen(const orc_cbs_params *p, double sigma_lwe, double sigma_rlwe, uint32_t qks, uint32_t base_ks,
                   uint64_t seed, int32_t *s_lwe, int32_t *s_rlwe, uint64_t *bsk, uint64_t *ht, uint64_t *ss,
                   uint16_t *ksk, uint64_t *tv, uint64_t *gpow, uint32_t *maps);
/* the grouped (mb = 2, 3 or 4) keys of the same key set: RGSW(prod_{i in S} s_i) per group and
 * key subset S (orc_mb_mask), [ceil(n/mb)][orc_mb_keys(mb)][2 digits_g][2][N]; one generator per group seeded
 * with seed ^ (0x9e3779b97f4a7c15 (g + 1)) */
void orc_cbs_keygen_mb(const orc_cbs_params *p, double sigma_rlwe, const int32_t *s_lwe, const int32_t *s_rlwe,
                       uint32_t mb, uint64_t seed, uint64_t *mbk);

/* ---------------- key generation on the device (cbs_keygen_device; no reference counterpart on
 * the device, the reference's keys come from its absent OpenFHE fork): every word from ChaCha20
 * under key[8], block (counter, nonce = (sample, domain, 0)): secrets domain 3 (s_lwe[i] = bit 0
 * of block (i, 0); s_rlwe[i] = floor(3 x / 2^128) - 1 of block (i, 1)), BSK domain 4 (sample
 * i 2 digits_g + row), HomTrace domain 5 (sample round digits_ht + j), SchemeSwitch domain 6,
 * KSK domain 7 (sample (j N + i) base_ks + v, mask words floor(qks x / 2^128) from block
 * (c, sample), noise from block (n, sample)), grouped keys domain 8 / 9 / 10 (mb = 2 / 3 / 4).
 * RLWE samples: NTT-domain mask floor(Q x / 2^128) of words 0-3, noise of words 4-5 by the
 * table of orc_cdt_table, b = a s + NTT(e); then the message as the seeded key generation adds
 * it.  Layouts as orc_cbs_keygen; any output may be NULL; returns 0 or -1 (no NTT tables). */
int orc_cbs_keygen_chacha(const orc_cbs_params *p, double sigma_lwe, double sigma_rlwe, uint32_t qks,
                          uint32_t base_ks, const uint32_t key[8], int32_t *s_lwe, int32_t *s_rlwe, uint64_t *bsk,
                          uint64_t *ht, uint64_t *ss, uint16_t *ksk);
void orc_cbs_keygen_chacha_mb(const orc_cbs_params *p, double sigma_rlwe, const uint32_t key[8],
                              const int32_t *s_lwe, const int32_t *s_rlwe, uint32_t mb, uint64_t *mbk);

/* ---------------- LMKCDEY blind rotation (bitwise/src/cirbts/cirbts-lmkcdey.cu; keys
 * cirbts-init.cu:630-726).  Powers: [0] = 2N - 5, then 5^i (i = 1 .. num_auto_keys), or for
 * window > 1 (the reference's CIRBTS_LMK_AUTOKEYS_WINDOW) 5^1 .. 5^window and 5^(2 window),
 * 5^(3 window), ... below 5^(N/2); maps [count][N] NTT-domain permutations out[t] = in[map[t]].
 * Keys: eval [n][2 digits_g][2][N] = RGSW(X^{s_i}), autok [count][digits_g][2][N] = RLWE(0)
 * with b -= 2^{g (j+1)} psi_k(s), both NTT domain, gadget powers 2^{g (j+1)} (the first
 * digit of the approximate decomposition is dropped).  orc_lmkcdey_eval_acc restates
 * LMKCDEY_EvalAcc on acc [2][N] in place for the negated masks a_neg mod 2N;
 * orc_blind_rotate_lmkcdey is the whole bootstrapping rotation (init, EvalAcc, finalize). */
uint32_t orc_lmkcdey_auto_pows(uint32_t N, uint32_t num_auto_keys, uint32_t window, uint32_t *pows);
void orc_lmkcdey_auto_maps(uint32_t N, uint32_t num_auto_keys, uint32_t window, uint32_t *maps);
void orc_lmkcdey_keygen(const orc_cbs_params *p, double sigma_rlwe, const int32_t *s_lwe, const int32_t *s_rlwe,
                        uint32_t num_auto_keys, uint32_t window, uint64_t seed, uint64_t *eval, uint64_t *autok);
void orc_lmkcdey_eval_acc(const orc_cbs_params *p, const uint64_t *eval, const uint64_t *autok, const uint32_t *maps,
                          uint32_t num_auto_keys, uint32_t window, const uint32_t *a_neg, uint32_t n, uint64_t *acc);
void orc_blind_rotate_lmkcdey(const orc_cbs_params *p, const orc_cbs_keys *k, const uint64_t *eval,
                              const uint64_t *autok, const uint32_t *maps, uint32_t num_auto_keys, uint32_t window,
                              const uint64_t *a, const uint64_t *b, uint32_t batch, uint32_t a_stride,
                              uint64_t *acc_out, int finalize);

#ifdef __cplusplus
}
#endif
#endif
