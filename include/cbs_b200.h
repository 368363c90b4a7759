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

#ifdef __cplusplus
}
#endif
#endif
