/*
 * cbs_b200.h -- C ABI of the B200-native bootstrapping hot path.
 *
 * One shared library (libcbs_b200.so) built for sm_100a.  Every entry point returns a
 * cbs_status; no C++ exception crosses this boundary.  On failure the message of the
 * calling thread's last error is available from cbs_last_error().
 *
 * Pointers named d_* are device pointers owned by the caller unless stated otherwise;
 * h_* are host pointers.  Streams are CUDA streams (cudaStream_t); NULL is the legacy
 * default stream.  A context is not thread-safe: use one per host thread (the reference's
 * GPUCirBTSContext has the same rule, bitwise/include/cirbts/cirbts.cuh:303-384).
 *
 * Each declaration names the reference interface it replaces (file:line relative to the
 * reference project root).
 */
#ifndef CBS_B200_H
#define CBS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *cbs_stream_t; /* == cudaStream_t */

typedef enum {
    CBS_OK = 0,
    CBS_ERR_INVALID_ARG = 1,
    CBS_ERR_SHAPE_MISMATCH = 2,
    CBS_ERR_OOM = 3,
    CBS_ERR_CUDA = 4,
    CBS_ERR_DEVICE_TIMEOUT = 5,
    CBS_ERR_UNSUPPORTED = 6,
    CBS_ERR_NOT_READY = 7
} cbs_status;

/* Message of the calling thread's most recent failure ("" if none). */
const char *cbs_last_error(void);
/* ABI version of this header (bumped on any signature change). */
int cbs_abi_version(void);

/* Device modulus record with the layout of Phantom's DModulus (include/ntt.cuh:9-37):
 * value and the Barrett constant floor(2^128 / value) as {low, high}. */
typedef struct {
    uint64_t value;
    uint64_t const_ratio[2];
} cbs_dmodulus;

/* ------------------------------------------------------------------------------------
 * Single-modulus negacyclic NTT, batched (Phantom 1-D).  Tables are Phantom's:
 * twiddles[N] / twiddles_shoup[N] = bit-reversed powers of the minimal primitive 2N-th
 * root and their Shoup quotients, itwiddles the inverse powers with N^-1 folded into
 * entry 1, scalar / scalar_shoup = N^-1 and its quotient (src/host/ntt.cu:11-56).
 * Supported dim: 1024, 2048, 4096.  Inputs fully reduced; outputs fully reduced.
 * ------------------------------------------------------------------------------------ */

/* replaces fnwt_1d_opt_batched (include/ntt.cuh:215; src/ntt/ntt_1d.cu:760) */
cbs_status cbs_fnwt_1d_opt_batched(uint64_t *d_inout, const uint64_t *d_twiddles, const uint64_t *d_twiddles_shoup,
                                   const cbs_dmodulus *d_modulus, size_t dim, size_t batch, cbs_stream_t stream);
/* out-of-place forward variant (no reference counterpart; same transform as above) */
cbs_status cbs_fnwt_1d_opt_outofplace_batched(uint64_t *d_out, const uint64_t *d_in, const uint64_t *d_twiddles,
                                              const uint64_t *d_twiddles_shoup, const cbs_dmodulus *d_modulus,
                                              size_t dim, size_t batch, cbs_stream_t stream);
/* replaces inwt_1d_opt_batched (include/ntt.cuh:219; src/ntt/ntt_1d.cu:767) */
cbs_status cbs_inwt_1d_opt_batched(uint64_t *d_inout, const uint64_t *d_itwiddles, const uint64_t *d_itwiddles_shoup,
                                   const cbs_dmodulus *d_modulus, const uint64_t *d_scalar,
                                   const uint64_t *d_scalar_shoup, size_t dim, size_t batch, cbs_stream_t stream);
/* replaces inwt_1d_opt_outofplace_batched (include/ntt.cuh:223; src/ntt/ntt_1d.cu:775) */
cbs_status cbs_inwt_1d_opt_outofplace_batched(uint64_t *d_out, const uint64_t *d_in, const uint64_t *d_itwiddles,
                                              const uint64_t *d_itwiddles_shoup, const cbs_dmodulus *d_modulus,
                                              const uint64_t *d_scalar, const uint64_t *d_scalar_shoup, size_t dim,
                                              size_t batch, cbs_stream_t stream);
/* replaces inwt_1d_opt_permute_batched (include/ntt.cuh:227; src/ntt/ntt_1d.cu:783):
 * slot i of each input reads in[map[i]] (negated when map[i] >= dim) before the INTT. */
cbs_status cbs_inwt_1d_opt_permute_batched(uint64_t *d_out, const uint64_t *d_in, const uint32_t *d_map,
                                           const uint64_t *d_itwiddles, const uint64_t *d_itwiddles_shoup,
                                           const cbs_dmodulus *d_modulus, const uint64_t *d_scalar,
                                           const uint64_t *d_scalar_shoup, size_t dim, size_t batch,
                                           cbs_stream_t stream);

/* Host helper: Phantom tables for (dim, q) into caller arrays (each dim words; n_inv: 2
 * words).  Replaces phantom::arith::NTT (src/host/ntt.cu:11-56) + DNTTTable upload. */
cbs_status cbs_ntt_tables_host(uint32_t dim, uint64_t q, uint64_t *h_twiddles, uint64_t *h_twiddles_shoup,
                               uint64_t *h_itwiddles, uint64_t *h_itwiddles_shoup, uint64_t *h_n_inv,
                               cbs_dmodulus *h_modulus);
/* Host helper: NTT-friendly primes, Phantom's search (src/host/numth.cu:207 get_primes). */
cbs_status cbs_get_primes(uint32_t ntt_size, int bit_size, uint32_t count, uint64_t *h_out);


/* ------------------------------------------------------------------------------------
 * Circuit bootstrapping context (replaces GPUCirBTSContext, bitwise/include/cirbts/
 * cirbts.cuh:31-500, and the OpenFHE CirBTS parameter / key objects it is built from).
 * ------------------------------------------------------------------------------------ */

typedef struct {
    uint32_t N;          /* RLWE ring dimension: 1024, 2048 or 4096 */
    uint64_t Q;          /* RLWE modulus: prime, Q = 1 mod 2N, Q < 2^62 */
    uint32_t n;          /* LWE dimension (blind-rotation steps) */
    uint64_t q_lwe;      /* LWE modulus of CBS inputs and key-switch outputs */
    uint32_t base_g;     /* blind-rotation gadget base (power of two), digitsG */
    uint32_t digits_g;
    uint32_t num_lut;    /* digitsCC: RGSW levels produced per bit (multi-value LUT count) */
    uint32_t base_cc;    /* RGSW / CMux gadget base (power of two) */
    uint32_t base_ht;    /* HomTrace key-switch gadget */
    uint32_t digits_ht;
    uint32_t base_ss;    /* SchemeSwitch gadget */
    uint32_t digits_ss;
    uint32_t trace_shift;/* log2 N - trace rounds; 0 = full trace */
    uint32_t qks;        /* extraction key-switch modulus (power of two, <= 2^16) */
    uint32_t base_ks;    /* extraction key-switch base (power of two, two digits cover qks) */
    double sigma_lwe;    /* noise of fresh LWE samples and of the key-switching key, [0, 1000) */
    double sigma_rlwe;   /* noise of RLWE / RGSW key material, [0, 1000) */
} cbs_params;

typedef struct cbs_context cbs_context;

/* The AES-128 parameter set of this build: N=2048, Q = 54-bit NTT prime, n=630, q=2^14,
 * BR gadget 2^12 x 3, RGSW out 2^6 x 4 (4 LUT levels), HomTrace 2^9 x 5, SchemeSwitch 2^9 x 5,
 * extraction KS qKS=2^14, base 2^7 (two digits). */
cbs_status cbs_params_default(cbs_params *out);
/* Named parameter sets.  CBS_PARAMS_AES_3X12 is cbs_params_default.  CBS_PARAMS_AES_2X18 is
 * the same set with the blind-rotation gadget 2^18 x 2 (18 low bits of Q still dropped): two
 * thirds of the external-product work and key bytes per blind-rotation step, for a larger
 * but still negligible decryption-failure probability (the noise budget of every other stage
 * is unchanged; the blind-rotation error reaches the RGSW rows only through the one
 * coefficient the trace keeps).  No reference counterpart: the reference's own sets live in
 * its absent OpenFHE fork (examples/aes_transcipher/main.cu:188-222). */
enum { CBS_PARAMS_AES_3X12 = 0, CBS_PARAMS_AES_2X18 = 1 };
cbs_status cbs_params_preset(int which, cbs_params *out);

/* replaces GPUCirBTSContext(const CirBTSContext&, uint32_t maxBatchSize) (cirbts.cuh:420)
 * plus gpu_init_ntt (cirbts-init.cu:867-1302): tables on the current device, scratch for
 * max_batch LWE inputs. */
cbs_status cbs_context_create(const cbs_params *params, uint32_t max_batch, cbs_context **out);
cbs_status cbs_context_destroy(cbs_context *ctx);
/* the context's compute stream (replaces GPUCirBTSContext::stream(), cirbts.cuh:452) */
cbs_status cbs_context_stream(const cbs_context *ctx, cbs_stream_t *out);

/* Generate all key material from a seed and upload it (replaces KeyGen, RLWEKeyGen,
 * CirBTKeyGen, KeySwitchGen at examples/aes_transcipher/main.cu:232-252, and
 * gpu_init_cirbsk, cirbts-init.cu:200-865). */
cbs_status cbs_keygen(cbs_context *ctx, uint64_t seed);

/* All key material generated on the device (no reference counterpart on the device: the
 * reference's KeyGen / CirBTKeyGen / KeySwitchGen run in its OpenFHE fork on the host,
 * examples/aes_transcipher/main.cu:232-252, and gpu_init_cirbsk re-lays the keys for the device
 * in host loops, bitwise/src/cirbts/cirbts-init.cu:367-864).  Every word comes from ChaCha20
 * (RFC 8439) under rng_key[32], one block per coefficient addressed by (counter, sample,
 * domain): secrets (domain 3), bootstrapping key (4), HomTrace keys (5), SchemeSwitch key (6),
 * extraction key-switching key (7), grouped keys when mb > 1 is selected (8 / 9 / 10); RLWE masks
 * in the NTT domain from words 0-3, noise from the discrete-Gaussian table of
 * cbs_cdt_table_host with words 4-5.  The same secrecy rules as cbs_aes128_setup_device apply:
 * rng_key decides the secret key, so it must come from a CSPRNG, stay secret and never be
 * reused; NULL draws a fresh key from the operating system (getrandom).  The context keeps
 * host copies (cbs_export_keys) and wipes its copy of rng_key on destroy. */
cbs_status cbs_keygen_device(cbs_context *ctx, const uint8_t *rng_key);

/* Blind-rotation external-product backend.  CBS_BR_NTT: exact 64-bit NTT arithmetic mod Q
 * (bit-identical to the reference's kernels).  CBS_BR_FFT64: FP64 FFT products (the
 * reference's gate-bootstrap / split-FFT form, bitwise/src/fft.cu:3614-3755); the key
 * spectra are precomputed from the keys, each product carries a bounded FP64 rounding error
 * that adds to the blind-rotation noise (the test suite states and checks the bound).
 * CBS_BR_FFT64_SPLIT: the reference's split-FFT CBS backend (CIRBTS_USE_SPLIT_FFT,
 * bitwise/src/cirbts/cirbts-init.cu:1084-1140, cirbts-bootstrap.cu:939-1085): the key is cut
 * into balanced limbs small enough that every FP64 digit x limb product rounds to its exact
 * integer, so the blind rotation -- and every output -- is bit-identical to CBS_BR_NTT's;
 * HomTrace, SchemeSwitch and the CMux run in their exact NTT forms.  GINX one-bit (2-4 gadget
 * digits) or grouped mb = 2 (2-3 digits, cbs_context_set_br_multibit after selecting the
 * backend), N = 1024 or 2048; CBS_ERR_UNSUPPORTED when no split of at most 4 limbs keeps the
 * products below 2^50 (cbs_split_fft_plan reports the split).  Selecting another backend resets
 * the grouping to mb = 1. */
enum { CBS_BR_NTT = 0, CBS_BR_FFT64 = 1, CBS_BR_FFT64_SPLIT = 2 };
cbs_status cbs_context_set_br_backend(cbs_context *ctx, int backend);

/* The limb split CBS_BR_FFT64_SPLIT uses for these parameters and grouping mb (1 or 2):
 * *limbs limbs of *limb_bits bits, every rounded limb-product coefficient below 2^*bound_bits
 * (<= 50).  The reference's sizing is limb_bits = 50 - (log2 Bg + log2 N + log2 digitsG2)
 * unsigned limbs (cirbts-init.cu:1097-1120); here the limbs are balanced and equalised, and
 * mb = 2 adds two bits for the monomial factor c0 + c1 + c0 c1.  CBS_ERR_UNSUPPORTED when no
 * split of at most 4 limbs exists. */
cbs_status cbs_split_fft_plan(const cbs_params *params, uint32_t mb, uint32_t *limbs, uint32_t *limb_bits,
                              uint32_t *bound_bits);

/* Multi-bit blind rotation (the reference's CIRBTS_PBS_MULTIBIT grouping,
 * bitwise/src/cirbts/cirbts-init.cu:376-565 and the MB3 MAC kernel.cu:4585-4771): mb = 1
 * processes one LWE coefficient per step (default); mb = 2 or 3 groups mb coefficients and
 * adds sum_S prod_{i in S}(X^{a_i} - 1) * (acc (x) RGSW(prod_{i in S} s_i)) over the
 * non-empty subsets S, so the accumulator is decomposed and transformed once per group.
 * mb = 4 is the reference's staged grouping (cirbts-batch.cu:2767-2923): groups of 4 with 8
 * keys ({0} {1} {2} {3} {0,1} {0,2} {1,2} {0,1,2}), applied as the mb = 3 step of coefficients
 * 0-2 and then a one-bit step of coefficient 3 on a fresh decomposition.  The grouped keys are
 * generated from the context's secrets (3, 7 or 8 RGSWs per group) when keys exist or are next
 * generated.  mb > 1 needs the FFT64 backend, or mb = 2 the split FFT backend
 * (CBS_ERR_UNSUPPORTED otherwise); selecting another backend resets mb to 1. */
cbs_status cbs_context_set_br_multibit(cbs_context *ctx, uint32_t mb);

/* Blind-rotation method (the reference's BINFHE_METHOD of the CirBTS context: GINX, or
 * LMKCDEY, bitwise/src/cirbts/cirbts-lmkcdey.cu:105-407 with keys cirbts-init.cu:630-726 and
 * the bootstrap cirbts-bootstrap.cu:600-720).  CBS_BR_LMKCDEY multiplies the accumulator by
 * RGSW(X^{s_i}) per coefficient with automorphisms X -> X^{5^k} (key switches) between
 * coefficients of different base-5 logarithm of their odd mask; num_auto_keys is the largest
 * power k with a key (the reference's numAutoKeys; keys for 2N - 5 and 5^1 .. 5^num_auto_keys).
 * window > 1 selects the reference's windowed key set (CIRBTS_LMK_AUTOKEYS_WINDOW,
 * cirbts-lmkcdey.cu:49-103, 311-325): keys for 2N - 5, 5^1 .. 5^window and 5^(2 window),
 * 5^(3 window), ... below 5^(N/2), a run of s steps closing with 5^(q window) then 5^r
 * (s = q window + r); window 0 or 1: non-windowed.  Its keys (RGSW(X^{s_i}) and the automorphism keys, approximate gadget with
 * powers 2^{g (j+1)}: the first g-bit digit is dropped, as the reference decomposes) are
 * generated from the context's secrets when keys exist or are next generated (seeded host
 * generator; for device-generated keys import them).  Preconditions, else CBS_ERR_UNSUPPORTED:
 * the NTT backend (selecting the FFT64 backend resets the method to GINX), g (digits_g + 1)
 * >= log2 Q (the 2^18 x 2 preset), and num_lut = 1: LMKCDEY rounds every mask to an odd
 * residue, which the multi-value test vector's rotations (multiples of 2^bitwidth) cannot
 * absorb (the reference's LMKCDEY path passes the masks unswitched and has the same limit).
 * The masks are rounded to Z_2N and forced odd (identical to the reference when q_lwe = 2N). */
enum { CBS_BR_GINX = 0, CBS_BR_LMKCDEY = 1 };
cbs_status cbs_context_set_br_method(cbs_context *ctx, int method, uint32_t num_auto_keys, uint32_t window);
/* The LMKCDEY keys, NTT domain: eval [n][2*digits_g][2][N] (RGSW(X^{s_i}); row 2j carries
 * 2^{g(j+1)} X^{s_i} on component a, row 2j+1 on b), autok [keys][digits_g][2][N] (RLWE(0) with
 * b -= 2^{g(j+1)} psi_k(s) for the key set's powers k in order: 2N - 5, 5^1, 5^2, ...).  Null
 * outputs: only the word counts are set. */
cbs_status cbs_export_lmkcdey_keys(const cbs_context *ctx, uint64_t *eval, uint64_t *autok, size_t *eval_words,
                                   size_t *auto_words);
/* Keys in the layout of cbs_export_lmkcdey_keys (a server without secrets); selects LMKCDEY
 * like cbs_context_set_br_method. */
cbs_status cbs_import_lmkcdey_keys(cbs_context *ctx, uint32_t num_auto_keys, uint32_t window, const uint64_t *eval,
                                   size_t eval_words, const uint64_t *autok, size_t auto_words);
/* Host-only generation of the LMKCDEY keys a context keyed with the same seed produces. */
cbs_status cbs_generate_lmkcdey_keys_host(const cbs_params *params, uint64_t seed, uint32_t num_auto_keys,
                                          uint32_t window, uint64_t *eval, uint64_t *autok, size_t *eval_words,
                                          size_t *auto_words);
/* NTT-domain automorphism maps [keys][N] of the key set (out[t] = in[map[t]] is X -> X^k in the
 * NTT domain; OpenFHE's PrecomputeAutoMap for this transform's slot order); *count (optional)
 * receives the number of keys; maps may be NULL. */
cbs_status cbs_lmkcdey_auto_maps_host(uint32_t N, uint32_t num_auto_keys, uint32_t window, uint32_t *maps,
                                      uint32_t *count);
/* LMKCDEY_EvalAcc (cirbts-lmkcdey.cu:105-407) on a batch, device pointers: a_neg [batch][a_stride]
 * the masks mod 2N as the reference's EvalAcc receives them (already negated by the caller,
 * cirbts-bootstrap.cu:681-689), acc [batch][2][N] NTT domain, updated in place.  One CTA per
 * ciphertext; the reference runs one ciphertext per call from the host. */
cbs_status cbs_lmkcdey_eval_acc_batch_device(cbs_context *ctx, const uint32_t *a_neg, uint32_t a_stride, uint64_t *acc,
                                             uint32_t batch, cbs_stream_t stream);
/* Schedule of the grouped FFT blind rotation with a two-digit gadget: CBS_BR_SCHEDULE_LOCKSTEP
 * transforms both digits of a polynomial together (interleaved butterflies, shared barriers),
 * CBS_BR_SCHEDULE_DIGITWISE one after the other, CBS_BR_SCHEDULE_PAIRED runs two ciphertexts per
 * CTA (mb = 2, N = 2048; 16 warps per SM, work split by output column);
 * CBS_BR_SCHEDULE_AUTO (default) takes the autotuner's cached choice for this GPU and parameter
 * set, else paired where it applies (mb = 2, N = 2048), else lockstep.  Results differ only by
 * FP64 rounding (all within the phase-error bound).  No reference counterpart. */
enum { CBS_BR_SCHEDULE_AUTO = 0, CBS_BR_SCHEDULE_DIGITWISE = 1, CBS_BR_SCHEDULE_LOCKSTEP = 2,
       CBS_BR_SCHEDULE_PAIRED = 3 };
cbs_status cbs_context_set_br_schedule(cbs_context *ctx, uint32_t schedule);

/* Autotuner of the blind rotation (no reference counterpart: the reference exposes ~70
 * environment knobs, examples/aes_transcipher/main.cu:107-136, and times three block sizes
 * inline, bitwise/src/cirbts/cirbts-batch.cu:2410-2460).  On the FFT64 backend it times the
 * blind rotation of `batch` synthetic LWE ciphertexts (CUDA events on the context's stream, one
 * warm-up and two timed launches per candidate) for every grouping mb in {1, 2, 3, 4} and, where
 * it applies, both schedules; grouped keys need the secret key (without it only the current mb
 * is timed).  The fastest is applied to the context and stored in the tuning cache under (GPU
 * name, parameter set, batch rounded up to a power of two): cache_path, or NULL for
 * $CBS_TUNE_CACHE, else $XDG_CACHE_HOME/cbs_b200/tune.json, else $HOME/.cache/cbs_b200/tune.json.
 * cbs_context_create reads the cache: a context whose mb was not set explicitly takes the
 * cached grouping when the FFT64 backend is selected, and its schedule at launch.
 * Synchronous; allocates; not for use inside a stream capture. */
typedef struct {
    uint32_t mb;             /* grouping of the blind rotation (1, 2, 3 or 4) */
    uint32_t schedule;       /* CBS_BR_SCHEDULE_DIGITWISE, _LOCKSTEP or _PAIRED */
    double us_per_bootstrap; /* measured at the tuned batch */
    uint32_t batch;          /* the batch the choice was measured at */
    uint32_t candidates;     /* configurations timed */
} cbs_tune_choice;
cbs_status cbs_autotune_blind_rotation(cbs_context *ctx, uint32_t batch, const char *cache_path, cbs_tune_choice *out);
/* The choice the context holds (from its cache read at creation or the last autotune);
 * CBS_ERR_NOT_READY when there is none. */
cbs_status cbs_context_tuned(const cbs_context *ctx, cbs_tune_choice *out);

/* The grouped keys of the current setting, NTT domain, for inspection and tests:
 * out [ceil(n/mb)][keys][2*digits_g][2][N] (null out: only *words is set; keys = 3, 7, 8 for
 * mb = 2, 3, 4), subsets in the order {0} {1} {2} {0,1} {0,2} {1,2} {0,1,2} (mb = 3),
 * {0} {1} {0,1} (mb = 2) or {0} {1} {2} {3} {0,1} {0,2} {1,2} {0,1,2} (mb = 4). */
cbs_status cbs_export_mb_bsk(const cbs_context *ctx, uint64_t *out, size_t *words);
/* Host-only generation of the grouped keys a context keyed with the same seed produces
 * (for CPU-side checks without a GPU); null out: only *words is set. */
cbs_status cbs_generate_mb_bsk_host(const cbs_params *params, uint64_t seed, uint32_t mb, uint64_t *out,
                                    size_t *words);

/* Export for verification (host buffers, NTT-domain normal form, reference layouts):
 * any pointer may be NULL.  s_lwe[n], s_rlwe[N]; bsk[n][2*digits_g][2][N];
 * ht[rounds][digits_ht][2][N]; ss[digits_ss][2][N]; ksk[2][N][base_ks][n+1];
 * tv[N] (coefficient domain); gpow[num_lut]; maps[rounds][N]. */
cbs_status cbs_export_keys(const cbs_context *ctx, int32_t *s_lwe, int32_t *s_rlwe, uint64_t *bsk, uint64_t *ht,
                           uint64_t *ss, uint16_t *ksk, uint64_t *tv, uint64_t *gpow, uint32_t *maps);

/* Load evaluation keys made elsewhere (by the key owner's cbs_generate_keys_host, or
 * cbs_export_keys of another context with the same parameters) instead of cbs_keygen: the
 * key upload of GPUCirBTSContext(const CirBTSContext&, maxBatch) (cirbts.cuh:420,
 * gpu_init_cirbsk cirbts-init.cu:200-865) for keys the caller owns.  bsk, ht, ss and ksk are
 * required, in the layouts of cbs_export_keys (every word checked: residues mod Q, KSK
 * entries below qks); the test vector, gadget powers and automorphism maps are derived from
 * the parameters.  The secrets are optional: with s_lwe = s_rlwe = NULL the context holds
 * evaluation keys only, and what needs a secret (generating grouped keys, cbs_aes128_setup,
 * cbs_lwe_decrypt_bits) returns CBS_ERR_NOT_READY; cbs_import_mb_bsk and
 * cbs_aes128_import_material then supply that material. */
cbs_status cbs_import_keys(cbs_context *ctx, const int32_t *s_lwe, const int32_t *s_rlwe, const uint64_t *bsk,
                           const uint64_t *ht, const uint64_t *ss, const uint16_t *ksk);
/* Grouped keys for mb = 2, 3 or 4 in the layout of cbs_export_mb_bsk (words must match);
 * selects mb like cbs_context_set_br_multibit.  FFT64 backend. */
cbs_status cbs_import_mb_bsk(cbs_context *ctx, uint32_t mb, const uint64_t *keys, size_t words);

/* The same key generation without a device (host buffers as in cbs_export_keys); the keys
 * of cbs_keygen(ctx, seed) equal those of cbs_generate_keys_host(params, seed). */
cbs_status cbs_generate_keys_host(const cbs_params *params, uint64_t seed, int32_t *s_lwe, int32_t *s_rlwe,
                                  uint64_t *bsk, uint64_t *ht, uint64_t *ss, uint16_t *ksk, uint64_t *tv,
                                  uint64_t *gpow, uint32_t *maps);

/* Device NTT tables of the context (replaces the accessors d_modulus() ... d_n_inv_mod_q_shoup(),
 * cirbts.cuh:431-455); any pointer may be NULL. */
cbs_status cbs_context_tables(const cbs_context *ctx, const cbs_dmodulus **d_modulus, const uint64_t **d_twiddles,
                              const uint64_t **d_twiddles_shoup, const uint64_t **d_itwiddles,
                              const uint64_t **d_itwiddles_shoup, const uint64_t **d_n_inv,
                              const uint64_t **d_n_inv_shoup);

/* Blind rotation + finalize + multi-value split for a batch of LWE ciphertexts
 * (replaces gpu_BootstrapLUT_inplace_batch_device, cirbts-batch.cu:3293-4629, and
 * kernel_GenMVRLWEs, kernel.cu:7498): d_a [batch][a_stride], d_b [batch] mod q_lwe ->
 * d_mv [batch][num_lut][2][N] NTT domain. */
cbs_status cbs_blind_rotate_batch_device(cbs_context *ctx, const uint64_t *d_a, const uint64_t *d_b, uint32_t batch,
                                         uint32_t a_stride, uint64_t *d_mv, cbs_stream_t stream);
/* HomTrace + SchemeSwitch for count MV RLWEs (cirbts-batch.cu:1628-1790):
 * d_mv [count][2][N] -> d_rgsw [count][2][2][N] (row 0 = scheme-switch row, row 1 = trace row). */
cbs_status cbs_trace_schemeswitch_device(cbs_context *ctx, const uint64_t *d_mv, uint32_t count, uint64_t *d_rgsw,
                                         cbs_stream_t stream);
/* Full batched circuit bootstrapping from device LWE (replaces
 * gpu_CircuitBootstrappingBatchToDeviceFromDeviceLWE, cirbts-batch.cu:1416-1879).
 * On success *d_rgsw_view points to context-owned [batch][num_lut][2][2][N] (layout
 * ((row*2+poly)*N + coeff) per bit, rows = 2*num_lut), valid until the next call that
 * reuses the context scratch (same contract as DeviceRGSWBatchView, cirbts.cuh:406-418). */
cbs_status cbs_circuit_bootstrap_batch_device(cbs_context *ctx, const uint64_t *d_a, const uint64_t *d_b,
                                              uint32_t batch, uint32_t a_stride, const uint64_t **d_rgsw_view,
                                              cbs_stream_t stream);

/* Host-buffer circuit bootstrapping (replaces gpu_CircuitBootstrappingBatch, cirbts-batch.cu:81,
 * and gpu_CircuitBootstrapping, cirbts-bootstrap.cu:89, whose OpenFHE LWECiphertext vectors
 * become plain arrays): h_a [batch][a_stride], h_b [batch] mod q_lwe (checked) ->
 * h_rgsw_out [batch][num_lut][2][2][N] (the layout of the device view), on the context's stream,
 * synchronous. */
cbs_status cbs_circuit_bootstrap_batch(cbs_context *ctx, const uint64_t *h_a, const uint64_t *h_b, uint32_t batch,
                                       uint32_t a_stride, uint64_t *h_rgsw_out);

/* Batched 8->32 CMux LUT (replaces EvalLUT8x32_RLWE_GPU_DeviceCtrl_Batch,
 * examples/aes_transcipher/gpu_lut.cuh:1783-2214): d_tables [tables][256][2][N] NTT domain,
 * h_table_of_lut[luts] selects the table, h_ctrl_bits[luts][8] indexes the control bit of
 * each tree level (bit 0 = LSB) in d_rgsw_all [bits][rgsw_stride]; d_out [luts][2][N]. */
cbs_status cbs_lut8x32_batch_device(cbs_context *ctx, const uint64_t *d_tables, uint32_t num_tables,
                                    const uint32_t *h_table_of_lut, const uint64_t *d_rgsw_all, uint32_t num_bits,
                                    uint64_t rgsw_stride, const uint32_t *h_ctrl_bits, uint32_t luts, uint64_t *d_out,
                                    cbs_stream_t stream);

/* One CMux per item (replaces one tree level of the reference's LUT, kernel_LUT_CMUX_Delta +
 * kernel_LUT_CMUX_ExternalProduct, examples/aes_transcipher/gpu_lut.cuh:521-595):
 * d_out[u] = d_ct0[u] + RGSW_u (x) (d_ct1[u] - d_ct0[u]) for u < count, RGSW_u the CBS output
 * rows of bit u at d_rgsw + u * rgsw_stride ([num_lut][2][2][N]; rgsw_stride = 0: one control for
 * every item, as at one level of a LUT tree); ciphertexts [count][2][N],
 * all NTT domain.  The context's backend picks the arithmetic: exact NTT products (CBS_BR_NTT)
 * or the FP64 FFT CMux of the AES path (CBS_BR_FFT64; inputs converted to the coefficient
 * domain and the rows to spectra inside the call, output back to the NTT domain). */
cbs_status cbs_cmux_batch_device(cbs_context *ctx, const uint64_t *d_ct0, const uint64_t *d_ct1,
                                 const uint64_t *d_rgsw, uint64_t rgsw_stride, uint32_t count, uint64_t *d_out,
                                 cbs_stream_t stream);

/* Sample extract + LWE key switch N->n + modulus switch qKS->q (replaces
 * ExtractStateBytesToLWEDeviceBatch, examples/aes_transcipher/extract.cuh:283-366, and
 * kernel_SampleExtractKeySwitchToLWE, aes_gpu_ks.cuh:538-607): d_words [words][2][N]
 * coefficient domain, h_info[count] = (word << 16) | coefficient; d_out_a [count][out_stride],
 * d_out_b [count] mod q_lwe. */
cbs_status cbs_extract_keyswitch_device(cbs_context *ctx, const uint64_t *d_words_coef, uint32_t words,
                                        const uint32_t *h_info, uint32_t count, uint64_t *d_out_a, uint64_t *d_out_b,
                                        uint32_t out_stride, cbs_stream_t stream);

/* ------------------------------------------------------------------------------------
 * Homomorphic AES-128 CTR transciphering (replaces the example's encrypted key material,
 * BuildEncryptedKeyMaterial key_material.cuh:12-46 + BuildTableRLWE rlwe_tables.cuh:17-24,
 * and the super-batch driver RunTranscipherBatch, examples/aes_transcipher/main.cu:1318-1619).
 * Output: per block 128 LWE ciphertexts (mod q_lwe, dimension n) of the AES-128 keystream
 * bits AES_K(counter), bit t = byte*8 + b (LSB first, byte in FIPS-197 state order).
 * ------------------------------------------------------------------------------------ */

/* Encrypt the AES material for key[16] under the context's keys (tables Te0..3/Te4_*, the
 * 11 round-key words, the round-0 key bits). */
cbs_status cbs_aes128_setup(cbs_context *ctx, const uint8_t *key, uint64_t seed);
/* The same material encrypted on the device (the reference encrypts it on the host, one
 * sample at a time: EncryptWord32RLWE / BuildTableRLWE, rlwe_tables.cuh:5-24;
 * BuildEncryptedKeyMaterial, key_material.cuh:12-46).  Randomness from ChaCha20 (RFC 8439)
 * under rng_key[32]: one block per coefficient, counter = coefficient index, nonce = (sample
 * index, 1 for RLWE / 2 for LWE, 0); masks floor(x q / 2^128) from words 0-3, noise from the
 * discrete Gaussian table of cbs_cdt_table_host with words 4-5.  Needs the secret key.
 * rng_key determines every mask and noise value, so it is as sensitive as the secret key:
 * whoever knows it recomputes (a, e) and solves b - e - m = a s for s, and two setups under
 * the same rng_key (another AES key, or another context sharing s) reveal the difference of
 * their messages.  It must come from a CSPRNG, stay secret and never be reused.  Pass
 * rng_key = NULL to have the call draw a fresh one from the operating system (getrandom);
 * a fixed rng_key is for reproducible tests only.  On any failure the context holds no AES
 * material (CBS_ERR_NOT_READY from the transcipher calls) until a setup succeeds. */
cbs_status cbs_aes128_setup_device(cbs_context *ctx, const uint8_t *key, const uint8_t *rng_key);
/* T[k] = floor(2^63 P(|X| <= k)) of the discrete Gaussian exp(-x^2 / 2 sigma^2), k = 0.. while
 * below 2^63; *len = its length; out (cap words) may be NULL to query the length. */
cbs_status cbs_cdt_table_host(double sigma, uint64_t *out, uint32_t cap, uint32_t *len);
/* Host copies of the encrypted material: tables [8][256][2][N], rk_words [11][4][2][N]
 * (NTT domain), rk0_a [128][n], rk0_b [128]; any pointer may be NULL. */
cbs_status cbs_aes128_export_material(const cbs_context *ctx, uint64_t *h_tables, uint64_t *h_rk_words,
                                      uint64_t *h_rk0_a, uint64_t *h_rk0_b);
/* Load encrypted material in the layouts above (made by the key owner's cbs_aes128_setup and
 * exported) instead of cbs_aes128_setup: a context holding evaluation keys only can then
 * transcipher; the AES key itself never reaches it.  Words checked (below Q / below q). */
cbs_status cbs_aes128_import_material(cbs_context *ctx, const uint64_t *h_tables, const uint64_t *h_rk_words,
                                      const uint64_t *h_rk0_a, const uint64_t *h_rk0_b);
/* Device variant: d_counter_bits [blocks*128] (0/1, bit t = byte*8 + b of each counter
 * block); d_out_a [blocks*128][n], d_out_b [blocks*128].  use_graphs != 0 replays one
 * captured CUDA graph per round (captured on the first call for a chunk size). */
cbs_status cbs_aes128_ctr_transcipher_device(cbs_context *ctx, const uint8_t *d_counter_bits, uint32_t blocks,
                                             uint64_t *d_out_a, uint64_t *d_out_b, int use_graphs,
                                             cbs_stream_t stream);
/* Host-buffer entry point: h_counters [blocks][16] -> h_out_a [blocks*128][n], h_out_b. */
cbs_status cbs_aes128_ctr_transcipher(cbs_context *ctx, const uint8_t *h_counters, uint32_t blocks,
                                      uint64_t *h_out_a, uint64_t *h_out_b);
/* Transciphering proper (replaces the per-bit EvalAddConstEq(ct, q/2) on the host after the
 * download, examples/aes_transcipher/main.cu:1569-1582): plaintext = keystream XOR public
 * AES-CTR ciphertext, so add q_lwe/2 (mod q_lwe) to d_b[t] wherever bit t of d_cipher
 * ([blocks][16] bytes, bit t = byte*8 + b, LSB first) is 1.  In place, on the device; d_b
 * (the keystream b words of cbs_aes128_ctr_transcipher_device) then encrypts the plaintext. */
cbs_status cbs_aes128_ctr_add_ciphertext_device(cbs_context *ctx, const uint8_t *d_cipher, uint32_t blocks,
                                                uint64_t *d_b, cbs_stream_t stream);
/* Host-buffer transciphering of a public AES-CTR ciphertext: h_counters and h_cipher
 * [blocks][16] -> h_out_a [blocks*128][n], h_out_b: LWE encryptions of the plaintext bits. */
cbs_status cbs_aes128_ctr_transcipher_ciphertext(cbs_context *ctx, const uint8_t *h_counters,
                                                 const uint8_t *h_cipher, uint32_t blocks, uint64_t *h_out_a,
                                                 uint64_t *h_out_b);
/* Client-side helper (uses the secret key): decrypt LWE bits (mod q_lwe) to 0/1. */
cbs_status cbs_lwe_decrypt_bits(const cbs_context *ctx, const uint64_t *h_a, const uint64_t *h_b, uint32_t count,
                                uint32_t a_stride, uint8_t *h_bits);

/* ------------------------------------------------------------------------------------
 * Circuit bootstrapping without device allocation.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc when they bootstrap: code inside a stream-capture
 * region (an allocation there breaks the capture), latency-bound serving loops (cudaMalloc /
 * cudaFree may synchronize the device), and components whose device memory belongs to
 * another allocator.  Same result as cbs_circuit_bootstrap_batch_device, but the caller
 * passes the output (d_rgsw_out [batch][num_lut][2][2][N]) and the blind-rotation ->
 * HomTrace hand-off lives in a fixed file-scope device array of
 * cbs_circuit_bootstrap_noalloc_capacity_words() 64-bit words (4 MiB; every GPU that loads
 * the library holds it until exit).  Batches with batch * num_lut * 2 * N above that are
 * rejected with CBS_ERR_SHAPE_MISMATCH (32 bits at N = 2048, num_lut = 4).  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress) and caches it:
 * make that first call before any stream capture.  All calls share the one array and it
 * keeps the last call's contents, so calls whose work overlaps on the GPU (different
 * streams or contexts in flight at once) race; serialize them.  The context itself must
 * already exist with its keys (cbs_context_create / cbs_keygen allocate). */
size_t cbs_circuit_bootstrap_noalloc_capacity_words(void);
/* The calling thread's current device must be the one the context was created on
 * (CBS_ERR_INVALID_ARG otherwise): the keys live there, and so does the array the call uses. */
cbs_status cbs_circuit_bootstrap_batch_device_noalloc(cbs_context *ctx, const uint64_t *d_a, const uint64_t *d_b,
                                                      uint32_t batch, uint32_t a_stride, uint64_t *d_rgsw_out,
                                                      cbs_stream_t stream);

/* ------------------------------------------------------------------------------------
 * Gate bootstrapping on the 32-bit torus: binfhe's GINX blind rotation with the FP64 FFT
 * external product, sample extract and LWE key switch (the reference's
 * GPUBinFHEContext::BatchGPUEvalBinGate path).  Torus values are uint32 (T = R/Z scaled by
 * 2^32); a bit is encrypted as +1/8 (1) or -1/8 (0).  LWE ciphertexts: a [count][n],
 * b [count].  Keys: s (LWE, binary, n), z (RLWE, binary, N); BSK [n][2*levels][2][N]
 * (RGSW(s_i), row 2k+p adds s_i * 2^(32-(k+1)*bg_bits) to component p of an RLWE(0) under z,
 * RLWE (a, b) with phase b - a*z); KSK [N][ks_levels][2^ks_base_bits - 1][n+1]
 * (LWE_s(v * z_i * 2^(32-(l+1)*ks_base_bits))).  The FFT products are exact after rounding
 * (|products| < 2^50), so results equal exact integer arithmetic.
 * ------------------------------------------------------------------------------------ */
typedef struct {
    uint32_t n;            /* LWE dimension */
    uint32_t N;            /* ring dimension: 1024 or 2048 */
    uint32_t bg_bits;      /* gadget base 2^bg_bits */
    uint32_t levels;       /* gadget digits (bg_bits * levels <= 30) */
    uint32_t ks_base_bits; /* key-switch base 2^ks_base_bits */
    uint32_t ks_levels;    /* key-switch digits */
    double sigma_lwe;      /* LWE and key-switch noise standard deviation on the torus */
    double sigma_rlwe;     /* bootstrapping-key noise standard deviation on the torus */
} cbs_gate_params;

/* gate codes (the first values of the reference's BINGATE; XOR / XNOR stand for both its
 * XOR_FAST / XNOR_FAST and XOR / XNOR, which binfhe-base-scheme-batch.cu:99-110 maps alike) */
enum { CBS_GATE_OR = 0, CBS_GATE_AND = 1, CBS_GATE_NOR = 2, CBS_GATE_NAND = 3, CBS_GATE_XOR = 4, CBS_GATE_XNOR = 5 };

typedef struct cbs_gate_context cbs_gate_context;

/* n = 636, N = 1024, base 2^7 x 3 digits, key switch base 2^2 x 8 digits, sigma_lwe = 2^-15,
 * sigma_rlwe = 2^-25 */
cbs_status cbs_gate_params_default(cbs_gate_params *out);
/* replaces GPUBinFHEContext construction + BTKeyGen (bitwise/include/binfhecontext.cuh) */
cbs_status cbs_gate_context_create(const cbs_gate_params *params, uint32_t max_batch, cbs_gate_context **out);
cbs_status cbs_gate_context_destroy(cbs_gate_context *ctx);
cbs_status cbs_gate_keygen(cbs_gate_context *ctx, uint64_t seed);
/* Grouped (multi-bit) blind rotation for the gate / ragged paths, the torus form of the
 * reference's CIRBTS_PBS_MULTIBIT grouping (bitwise/src/cirbts/cirbts-init.cu:376-530): mb = 1
 * (default) or 2 / 3; the grouped keys RGSW_z(prod_{i in S} s_i) are generated from the
 * context's secrets (now, or at the next cbs_gate_keygen).  cbs_gate_export_mb_bsk returns them
 * [ceil(n/mb)][2^mb - 1][2*levels][2][N] (null out: only *words). */
cbs_status cbs_gate_set_multibit(cbs_gate_context *ctx, uint32_t mb);
cbs_status cbs_gate_export_mb_bsk(const cbs_gate_context *ctx, uint32_t *out, size_t *words);
/* Arithmetic of the external product in the gate / ragged blind rotation:
 *   CBS_FFT_FP64        FP64 transforms; every product rounds to the exact integer (default);
 *   CBS_FFT_FP32_SPLIT  FP32 transforms, keys split k = lo + 2^S hi (S = log2 N + 14: a 24- or
 *                       25-bit lo and a 7- or 8-bit hi limb), recombined in integers; the hi
 *                       limb is exact, the lo limb leaves ~2^11 rms of FP32 error per product
 *                       on the 2^32 torus;
 *   CBS_FFT_FP32        FP32 transforms on the whole key (~2^19 rms per product; the phase
 *                       error of a bootstrap then reaches the gate margin: comparison only).
 * The FP32 modes need mb = 1; split FP32 needs bg_bits <= 7.
 * This is the limb split of the reference's split-FFT backend (bitwise/src/cirbts/
 * cirbts-init.cu:1084-1140, FP64 there) in FP32 on the 32-bit torus. */
enum { CBS_FFT_FP64 = 0, CBS_FFT_FP32_SPLIT = 1, CBS_FFT_FP32 = 2 };
cbs_status cbs_gate_set_fft_mode(cbs_gate_context *ctx, uint32_t mode);
/* the same keys as cbs_gate_keygen(ctx, seed) on the host only (no device); NULL skips */
cbs_status cbs_gate_generate_keys_host(const cbs_gate_params *params, uint64_t seed, int32_t *s_lwe, int32_t *z_rlwe,
                                       uint32_t *bsk, uint32_t *ksk);
/* host copies of the secrets and keys (any pointer may be NULL) */
cbs_status cbs_gate_export_keys(const cbs_gate_context *ctx, int32_t *s_lwe, int32_t *z_rlwe, uint32_t *bsk,
                                uint32_t *ksk);
/* host-side encryption / decryption of bits under s (test and setup helpers) */
cbs_status cbs_gate_encrypt_bits(const cbs_gate_context *ctx, const uint8_t *h_bits, uint32_t count, uint64_t seed,
                                 uint32_t *h_a, uint32_t *h_b);
cbs_status cbs_gate_decrypt_bits(const cbs_gate_context *ctx, const uint32_t *h_a, const uint32_t *h_b,
                                 uint32_t count, uint8_t *h_bits);
/* replaces GPUBinFHEContext::BatchGPUEvalBinGate (bitwise/include/binfhecontext.cuh:53-57;
 * bitwise/src/binfhe-base-scheme-batch.cu:82-200): out_k = gate(in1_k, in2_k) for k < count */
cbs_status cbs_gate_eval_batch_device(cbs_gate_context *ctx, int gate, const uint32_t *d_a1, const uint32_t *d_b1,
                                      const uint32_t *d_a2, const uint32_t *d_b2, uint32_t count, uint32_t *d_out_a,
                                      uint32_t *d_out_b, cbs_stream_t stream);
/* the bootstrap alone (sign: +1/8 when the phase is in [0, 1/2), else -1/8), with the
 * extracted LWE of dimension N ([count][N+1], a then b) written to d_ext when non-NULL
 * (BatchGPUBootstrapGateCore + sample extract, binfhe-base-scheme-batch.cu:16-140) */
cbs_status cbs_gate_bootstrap_batch_device(cbs_gate_context *ctx, const uint32_t *d_a, const uint32_t *d_b,
                                           uint32_t count, uint32_t *d_ext, uint32_t *d_out_a, uint32_t *d_out_b,
                                           cbs_stream_t stream);

/* Functional bootstrapping on the gate context (the reference's large-precision evaluators,
 * https://eprint.iacr.org/2021/1337, as bitwise/src/binfhe-base-scheme-batch.cu:215-712 batches
 * them behind GPUBinFHEContext::BatchGPUEvalFunc / Floor / Sign / Decomp,
 * bitwise/include/binfhecontext.cuh:60-118).  Ciphertexts here are LWE vectors under the
 * context's key s with an explicit power-of-two modulus, as the reference's LWECiphertext
 * carries one: a [count][n], b [count], uint32 words holding residues mod that modulus (device
 * pointers).  The bootstraps need the FP64 external product (cbs_gate_set_fft_mode) and allocate
 * the context's scratch on first use.  beta is the reference's GetBeta() (OpenFHE's error bound,
 * 128 in its parameter sets), q its LWE modulus Getq() (a power of two dividing 2N).
 *
 * cbs_gate_bootstrap_func_batch_device: BatchGPUBootstrapFunc (:215-364): input mod q_in
 * (power of two, 4 <= q_in <= 2N), f given on [0, q_in/2) by h_lut [q_in/2] (host, values in
 * [0, fmod)); the output (mod fmod, a power of two <= 2^32) encrypts f(phase) for phases in
 * [0, q_in/2) and -f(phase - q_in/2) above (the negacyclic extension every caller relies on). */
cbs_status cbs_gate_bootstrap_func_batch_device(cbs_gate_context *ctx, const uint32_t *d_a, const uint32_t *d_b,
                                                uint32_t count, uint32_t q_in, const uint64_t *h_lut, uint64_t fmod,
                                                uint32_t *d_out_a, uint32_t *d_out_b, cbs_stream_t stream);
/* BatchGPUEvalFunc (:366-479): ciphertexts mod q (power of two <= 2N), h_lut [q] (host, values
 * mod q) the function on Z_q; negacyclic tables take one bootstrap, periodic ones two, any
 * other table (q <= N) two at modulus 2q.  Output mod q. */
cbs_status cbs_gate_eval_func_batch_device(cbs_gate_context *ctx, const uint32_t *d_a, const uint32_t *d_b,
                                           uint32_t count, uint32_t q, const uint32_t *h_lut, uint32_t beta,
                                           uint32_t *d_out_a, uint32_t *d_out_b, cbs_stream_t stream);
/* BatchGPUEvalFloor (:481-543): ciphertexts mod `mod` (power of two <= 2^32); clears the low
 * bits of the phase below q (roundbits = 0) or below beta 2^(roundbits+1); output mod `mod`. */
cbs_status cbs_gate_eval_floor_batch_device(cbs_gate_context *ctx, const uint32_t *d_a, const uint32_t *d_b,
                                            uint32_t count, uint64_t mod, uint32_t q, uint32_t roundbits,
                                            uint32_t beta, uint32_t *d_out_a, uint32_t *d_out_b, cbs_stream_t stream);
/* BatchGPUEvalSign (:545-631): ciphertexts mod `mod` > q; floors and switches the modulus down
 * by q / (2 beta) until it is at most q, then bootstraps the sign: output mod q encrypting 0
 * for phases below mod/2 and q/2 above (scheme_switch: -q/4 and q/4, the reference's encoding
 * for scheme switching).  Its single bootstrapping key serves every round (the reference's GPU
 * context holds one, so its base-switching branch never runs). */
cbs_status cbs_gate_eval_sign_batch_device(cbs_gate_context *ctx, const uint32_t *d_a, const uint32_t *d_b,
                                           uint32_t count, uint64_t mod, uint32_t q, uint32_t beta, int scheme_switch,
                                           uint32_t *d_out_a, uint32_t *d_out_b, cbs_stream_t stream);
/* BatchGPUEvalDecomp (:633-712): ciphertexts mod `mod` > q into digits, least significant first:
 * digit k [k][count][n] / [k][count] is the phase mod q before the k-th floor, the last the
 * remainder at the final modulus.  *digits: in, the capacity of the outputs; out, the digits
 * made (also when the capacity is too small, CBS_ERR_INVALID_ARG). */
cbs_status cbs_gate_eval_decomp_batch_device(cbs_gate_context *ctx, const uint32_t *d_a, const uint32_t *d_b,
                                             uint32_t count, uint64_t mod, uint32_t q, uint32_t beta,
                                             uint32_t *d_out_a, uint32_t *d_out_b, uint32_t *digits,
                                             cbs_stream_t stream);

/* Ragged batching: many bootstrap requests of uneven size (the sign bootstrap of
 * cbs_gate_bootstrap_batch_device, outputs key-switched to n) in one blind-rotation launch
 * and one key-switch launch per parameter set, instead of one launch pair per request.  No
 * reference counterpart (the reference launches per batch).  cbs_gate_ragged_plan uploads
 * the request table and sizes the context's scratch (synchronous; call it outside any
 * stream capture); grid_ctas bounds the blind rotation's grid (0: one CTA per ciphertext;
 * smaller grids make each CTA loop over ciphertexts).  cbs_gate_ragged_launch only launches
 * kernels, so it can be captured in a CUDA graph and replayed; each replay reruns the plan
 * on whatever the planned buffers then hold.  Contexts of different parameter sets launch
 * their plans on separate streams to run side by side. */
typedef struct {
    const uint32_t *d_a; /* [count][n] */
    const uint32_t *d_b; /* [count] */
    uint32_t *d_out_a;   /* [count][n] */
    uint32_t *d_out_b;   /* [count] */
    uint32_t count;
} cbs_gate_request;
cbs_status cbs_gate_ragged_plan(cbs_gate_context *ctx, const cbs_gate_request *h_reqs, uint32_t num_reqs,
                                uint32_t grid_ctas);
cbs_status cbs_gate_ragged_launch(cbs_gate_context *ctx, cbs_stream_t stream);
/* Picks the persistent grid of the current plan (the ragged launch's tile schedule): times one
 * ragged launch per candidate (one CTA per ciphertext, 2, 4 and 8 CTAs per SM) with CUDA
 * events, keeps the fastest in the plan and returns it (and its time in ms; either pointer may
 * be NULL).  Runs the plan's launches, so the planned outputs are overwritten; synchronous, not
 * for use inside a stream capture.  No reference counterpart. */
cbs_status cbs_gate_ragged_autotune(cbs_gate_context *ctx, uint32_t *chosen_grid, double *ms);

/* ------------------------------------------------------------------------------------
 * Torus circuit bootstrapping with private functional key switching (PFKS): an LWE bit
 * (level 0: dimension n, torus32) becomes an RGSW ciphertext under a level-1 RLWE key
 * (N1, torus32) through cb_levels level-2 blind rotations (ring N2, 64-bit torus, gadget
 * 2^bg2_bits x l2, FP64 FFT products) with the test vectors g_k / 2, g_k = 2^-(cb_bits (k+1)),
 * and two PFKS per level (digits of the top 32 bits) into RLWE rows:
 * row 2k+1 = PFKS_id(m g_k) (component b carries m g_k), row 2k = PFKS_{-z1}(m g_k)
 * (component a carries m g_k).  No counterpart in the reference, whose circuit bootstrap
 * uses HomTrace + SchemeSwitch (cbs_circuit_bootstrap_batch_device); this is the PFKS
 * form the configuration names (base 2^4, 8 digits).  Output RGSW:
 * [count][cb_levels][2 rows][2 polys][N1] u32, row 2k+c with the message on component c.
 * Keys: level-2 BSK [n][2*l2][2][N2] uint64; PFKS [2 functions (-z1, id)][N2+1][pfks_levels]
 * [2^pfks_base_bits - 1][2][N1] uint32.
 * ------------------------------------------------------------------------------------ */
typedef struct {
    uint32_t n;              /* level-0 LWE dimension */
    uint32_t N2;             /* level-2 ring (blind rotation): 1024 or 2048 on the device */
    uint32_t bg2_bits, l2;   /* level-2 gadget */
    uint32_t N1;             /* level-1 ring (output RGSW) */
    uint32_t cb_bits, cb_levels;          /* output RGSW gadget (cb_levels <= 8) */
    uint32_t pfks_base_bits, pfks_levels; /* PFKS digits (base_bits * levels = 32) */
    double sigma_lwe;        /* level-0 noise */
    double sigma_lvl2;       /* level-2 bootstrapping-key noise */
    double sigma_lvl1;       /* PFKS key noise */
} cbs_tcb_params;

typedef struct cbs_tcb_context cbs_tcb_context;

/* n = 630, N2 = 2048, 2^9 x 3, N1 = 1024, output 2^6 x 3, PFKS 2^4 x 8, sigma 2^-15 / 2^-44 / 2^-25 */
cbs_status cbs_tcb_params_default(cbs_tcb_params *out);
cbs_status cbs_tcb_context_create(const cbs_tcb_params *params, uint32_t max_batch, cbs_tcb_context **out);
cbs_status cbs_tcb_context_destroy(cbs_tcb_context *ctx);
cbs_status cbs_tcb_keygen(cbs_tcb_context *ctx, uint64_t seed);
/* Grouped level-2 blind rotation (mb = 1, 2 or 3), as cbs_gate_set_multibit; keys on the
 * 64-bit torus, [ceil(n/mb)][2^mb - 1][2*l2][2][N2]. */
cbs_status cbs_tcb_set_multibit(cbs_tcb_context *ctx, uint32_t mb);
cbs_status cbs_tcb_export_mb_bsk(const cbs_tcb_context *ctx, uint64_t *out, size_t *words);
/* the same keys on the host only (no device); NULL skips an output */
cbs_status cbs_tcb_generate_keys_host(const cbs_tcb_params *params, uint64_t seed, int32_t *s0, int32_t *z2,
                                      int32_t *z1, uint64_t *bsk2, uint32_t *pfks);
cbs_status cbs_tcb_export_keys(const cbs_tcb_context *ctx, int32_t *s0, int32_t *z2, int32_t *z1, uint64_t *bsk2,
                               uint32_t *pfks);
cbs_status cbs_tcb_encrypt_bits(const cbs_tcb_context *ctx, const uint8_t *h_bits, uint32_t count, uint64_t seed,
                                uint32_t *h_a, uint32_t *h_b);
/* d_a [count][n], d_b [count] -> d_rgsw [count][cb_levels][2][2][N1]; d_ext (optional,
 * [count][cb_levels][N2+1] uint64) receives the level-2 LWEs of m g_k that feed the PFKS */
cbs_status cbs_tcb_circuit_bootstrap_device(cbs_tcb_context *ctx, const uint32_t *d_a, const uint32_t *d_b,
                                            uint32_t count, uint64_t *d_ext, uint32_t *d_rgsw, cbs_stream_t stream);

/* ------------------------------------------------------------------------------------
 * RNS (Phantom) core: multi-prime NTT and hybrid key switching, CKKS form.
 * Key modulus chain = the size_q primes of Q followed by the size_p special primes P
 * (every one < 2^60, prime, = 1 mod 2N, distinct); alpha = size_p is the digit width and
 * a level-l ciphertext (size_ql = l limbs of Q) has beta = ceil(l / alpha) digits.
 * Layouts (uint64 residues, NTT domain, limb-major):
 *   c2 [count][size_ql][N]; ciphertext polys ct [count][2][size_ql][N];
 *   t_mod_up [count][beta][size_ql + size_p][N]; cx [count][2][size_ql + size_p][N];
 *   evk of digit b: [2][size_q + size_p][N] (component 0 then 1, key-chain limbs).
 * All outputs are fully reduced and equal to the reference's bit for bit.
 * ------------------------------------------------------------------------------------ */
typedef struct cbs_rns_context cbs_rns_context;

/* Device tables of the whole chain with the layout of Phantom's DNTTTable
 * (include/ntt.cuh:100-160): [size][n] power tables, [size] n^-1, [size] moduli. */
typedef struct {
    const uint64_t *twiddle, *twiddle_shoup, *itwiddle, *itwiddle_shoup, *n_inv, *n_inv_shoup;
    const cbs_dmodulus *modulus;
    uint32_t n, size;
} cbs_rns_ntt_tables;

/* replaces PhantomContext(const EncryptionParameters&) for the key-switching path
 * (include/context.cuh:161; src/context.cu): poly_degree 2^10 .. 2^17, 1 <= size_p <= 16,
 * size_q + size_p <= 256 */
cbs_status cbs_rns_context_create(uint32_t poly_degree, const uint64_t *h_q, uint32_t size_q, const uint64_t *h_p,
                                  uint32_t size_p, cbs_rns_context **out);
cbs_status cbs_rns_context_destroy(cbs_rns_context *ctx);
/* Device fault word of the RNS context: bit CBS_RNS_FAULT_BULK_COPY is set when a bulk copy of
 * the FP64-pipe transforms did not complete within its bounded wait (about a second); the
 * launch then finishes with unreliable outputs instead of hanging.  Synchronizes the device;
 * clear != 0 resets the word.  0 after every correct run.  No reference counterpart. */
enum { CBS_RNS_FAULT_BULK_COPY = 1 };
cbs_status cbs_rns_device_fault(cbs_rns_context *ctx, uint32_t *out, int clear);
/* replaces PhantomContext::gpu_rns_tables() (include/context.cuh) */
cbs_status cbs_rns_context_tables(const cbs_rns_context *ctx, cbs_rns_ntt_tables *out);
/* Builds (once) the modup / moddown constants of level size_ql; the other calls build them on
 * first use with synchronous copies, so call this first when the later calls are captured
 * into a CUDA graph.  No reference counterpart (the reference builds every level in the
 * PhantomContext constructor, src/context.cu). */
cbs_status cbs_rns_prepare_level(cbs_rns_context *ctx, uint32_t size_ql);
/* replaces nwt_2d_radix8_forward_inplace / nwt_2d_radix8_backward_inplace (include/ntt.cuh:232,
 * :262; src/ntt/fntt_2d.cu:620, intt_2d.cu:724): limbs start .. start + size - 1 of the chain,
 * limb i at d_inout + i * N (d_inout is the base of the whole polynomial, as in the reference) */
cbs_status cbs_nwt_2d_radix8_forward_inplace(cbs_rns_context *ctx, uint64_t *d_inout, uint32_t coeff_modulus_size,
                                             uint32_t start_modulus_idx, cbs_stream_t stream);
cbs_status cbs_nwt_2d_radix8_backward_inplace(cbs_rns_context *ctx, uint64_t *d_inout, uint32_t coeff_modulus_size,
                                              uint32_t start_modulus_idx, cbs_stream_t stream);
/* Batched form of the two above: polys polynomials poly_stride words apart, each holding
 * coeff_modulus_size limbs (chain primes start ..) contiguously from its first word.  No
 * reference counterpart (the reference loops over polynomials). */
cbs_status cbs_rns_ntt_batched(cbs_rns_context *ctx, uint64_t *d_data, uint32_t polys, uint64_t poly_stride,
                               uint32_t coeff_modulus_size, uint32_t start_modulus_idx, int inverse,
                               cbs_stream_t stream);
/* replaces DRNSTool::modup (include/rns.cuh:156; src/rns_bconv.cu:530-634), CKKS form, for
 * count ciphertexts at once: d_c2 [count][size_ql][N] -> d_t_mod_up [count][beta][size_ql+size_p][N] */
cbs_status cbs_rns_modup(cbs_rns_context *ctx, uint64_t *d_t_mod_up, const uint64_t *d_c2, uint32_t size_ql,
                         uint32_t count, cbs_stream_t stream);
/* replaces key_switch_inner_prod_c2_and_evk (src/eval_key_switch.cu:13-68): h_evks is a host
 * array of beta device pointers (PhantomRelinKey::public_keys_ptr(), one key per digit) */
cbs_status cbs_rns_key_switch_inner_prod(cbs_rns_context *ctx, uint64_t *d_cx, const uint64_t *d_t_mod_up,
                                         const uint64_t *const *h_evks, uint32_t size_ql, uint32_t count,
                                         cbs_stream_t stream);
/* replaces DRNSTool::moddown_from_NTT (include/rns.cuh:162; src/rns_bconv.cu:776-828), CKKS
 * form, for polys polynomials: d_cx [polys][size_ql+size_p][N] -> d_ct [polys][size_ql][N];
 * accumulate != 0 adds the result to d_ct (the add_to_ct step of keyswitch_inplace).  The P
 * limbs of d_cx are overwritten (scratch), as in the reference. */
cbs_status cbs_rns_moddown_from_ntt(cbs_rns_context *ctx, uint64_t *d_ct, uint64_t *d_cx, uint32_t size_ql,
                                    uint32_t polys, int accumulate, cbs_stream_t stream);
/* replaces keyswitch_inplace(const PhantomContext&, PhantomCiphertext&, uint64_t *c2,
 * const PhantomRelinKey&, bool, const cudaStream_t&) (include/evaluate.cuh:29;
 * src/eval_key_switch.cu:94-181), CKKS form, for count ciphertexts: d_ct [count][2][size_ql][N]
 * += keyswitch(d_c2 [count][size_ql][N]).  Scratch is held by the context. */
cbs_status cbs_rns_keyswitch_inplace(cbs_rns_context *ctx, uint64_t *d_ct, const uint64_t *d_c2,
                                     const uint64_t *const *h_evks, uint32_t size_ql, uint32_t count,
                                     cbs_stream_t stream);

/* ---- CKKS evaluator on the RNS context (src/evaluate.cu; csrc/ckks.cu) ----
 * Ciphertexts are NTT-domain polynomials over the first size_ql primes of the chain,
 * [size][size_ql][N] (PhantomCiphertext::data(): size 2, or 3 after a multiplication); all
 * outputs fully reduced.  Key arrays are host arrays of beta device pointers, as for
 * cbs_rns_keyswitch_inplace. */
/* replaces add_inplace (include/evaluate.cuh:46): ct1 += ct2 over size polynomials */
cbs_status cbs_ckks_add_inplace(cbs_rns_context *ctx, uint64_t *d_ct1, const uint64_t *d_ct2, uint32_t size,
                                uint32_t size_ql, cbs_stream_t stream);
/* replaces sub_inplace (include/evaluate.cuh:61): ct1 = ct1 - ct2, or ct2 - ct1 when negate */
cbs_status cbs_ckks_sub_inplace(cbs_rns_context *ctx, uint64_t *d_ct1, const uint64_t *d_ct2, uint32_t size,
                                uint32_t size_ql, int negate, cbs_stream_t stream);
/* replaces negate_inplace (include/evaluate.cuh:37) */
cbs_status cbs_ckks_negate_inplace(cbs_rns_context *ctx, uint64_t *d_ct, uint32_t size, uint32_t size_ql,
                                   cbs_stream_t stream);
/* replaces multiply_plain_inplace (include/evaluate.cuh:94), CKKS: every polynomial times the
 * NTT-domain plaintext d_plain [size_ql][N] */
cbs_status cbs_ckks_multiply_plain_inplace(cbs_rns_context *ctx, uint64_t *d_ct, const uint64_t *d_plain,
                                           uint32_t size, uint32_t size_ql, cbs_stream_t stream);
/* replaces multiply_inplace (include/evaluate.cuh:105; bgv_ckks_multiply, src/evaluate.cu:345):
 * d_ct1 [3][size_ql][N] holds (a0, a1) on entry and (a0 b0, a0 b1 + a1 b0, a1 b1) on return;
 * d_ct2 = (b0, b1), or d_ct1 itself to square; other overlaps are rejected */
cbs_status cbs_ckks_multiply_inplace(cbs_rns_context *ctx, uint64_t *d_ct1, const uint64_t *d_ct2, uint32_t size_ql,
                                     cbs_stream_t stream);
/* replaces relinearize_inplace (include/evaluate.cuh:125; src/evaluate.cu:1345): d_ct
 * [3][size_ql][N] -> its first two polynomials += keyswitch(c2) with the relinearisation key */
cbs_status cbs_ckks_relinearize_inplace(cbs_rns_context *ctx, uint64_t *d_ct, const uint64_t *const *h_relin_keys,
                                        uint32_t size_ql, cbs_stream_t stream);
/* replaces multiply_and_relin_inplace (include/evaluate.cuh:115) */
cbs_status cbs_ckks_multiply_and_relin_inplace(cbs_rns_context *ctx, uint64_t *d_ct1, const uint64_t *d_ct2,
                                               const uint64_t *const *h_relin_keys, uint32_t size_ql,
                                               cbs_stream_t stream);
/* replaces rescale_to_next (include/evaluate.cuh:137; DRNSTool::divide_and_round_q_last_ntt,
 * src/rns.cu:1183-1208): d_src [size][size_ql][N] -> d_dst [size][size_ql - 1][N]; d_src is
 * left unchanged (the reference works on a copy) */
cbs_status cbs_ckks_rescale_to_next(cbs_rns_context *ctx, uint64_t *d_dst, const uint64_t *d_src, uint32_t size,
                                    uint32_t size_ql, cbs_stream_t stream);
/* replaces mod_switch_to_next (include/evaluate.cuh:146), CKKS: drop the last limb */
cbs_status cbs_ckks_mod_switch_to_next(cbs_rns_context *ctx, uint64_t *d_dst, const uint64_t *d_src, uint32_t size,
                                       uint32_t size_ql, cbs_stream_t stream);
/* replaces phantom::util::get_elt_from_step (include/galois.cuh:17): the Galois element of a
 * rotation by step slots (0 = conjugation); 0 when |step| >= N/2 */
uint32_t cbs_ckks_galois_elt_from_step(int step, uint32_t poly_degree);
/* replaces apply_galois_inplace (include/evaluate.cuh:215; src/evaluate.cu:1571), CKKS: the
 * NTT-slot permutation of the element on both polynomials, then c1 wiped and
 * (c0, 0) += keyswitch(sigma(c1)) with the element's Galois key.  d_ct [2][size_ql][N]. */
cbs_status cbs_ckks_apply_galois_inplace(cbs_rns_context *ctx, uint64_t *d_ct, uint32_t galois_elt,
                                         const uint64_t *const *h_galois_keys, uint32_t size_ql, cbs_stream_t stream);
/* replaces rotate_inplace (include/evaluate.cuh:229) */
cbs_status cbs_ckks_rotate_inplace(cbs_rns_context *ctx, uint64_t *d_ct, int step, const uint64_t *const *h_galois_keys,
                                   uint32_t size_ql, cbs_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif
