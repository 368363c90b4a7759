// ckks.cu -- CKKS evaluator operations on the RNS (Phantom-core) context: the NTT-domain
// arithmetic of src/evaluate.cu on top of this library's 2-D NTT and hybrid key switching.
//
// Ciphertexts are NTT-domain polynomials of size_ql limbs, [size][size_ql][N] (size 2, or 3
// after a multiplication), the layout of PhantomCiphertext::data().  Follows:
//   add_inplace / sub_inplace / negate_inplace   src/evaluate.cu (add_rns_poly, sub_rns_poly,
//                                                negate_rns_poly, polymath.cu)
//   multiply_plain_inplace                       multiply_rns_poly (per limb, CKKS branch)
//   multiply_inplace (bgv_ckks_multiply)         tensor_prod_2x2_rns_poly / tensor_square_2x2
//   relinearize_inplace                          keyswitch of c2 with the relinearisation key
//   rescale_to_next                              DRNSTool::divide_and_round_q_last_ntt
//                                                (src/rns.cu:1183-1208): INTT of the last limb,
//                                                its residues mod every other prime, NTT, then
//                                                (c_j - that) q_last^-1 mod q_j
//   mod_switch_to_next                           drop the last limb (mod_switch_drop_to_next)
//   apply_galois_inplace / rotate_inplace        PhantomGaloisTool permutation of the NTT
//                                                slots (include/galois.cuh:78-91) and a keyswitch
//                                                of sigma(c1) with the Galois key, c1 wiped
// Element-wise products use the exact FP64 form (fp64_mod.cuh) when every prime is below 2^50
// and 128-bit products with Barrett reduction otherwise; every result is the fully reduced
// residue, the reference's words.
#include <cstring>
#include <memory>
#include <vector>

#include "arith.cuh"
#include "common.cuh"
#include "fp64_mod.cuh"
#include "rns_context.cuh"

namespace cbs {

namespace {

constexpr uint32_t kCkksThreads = 256;

struct ElemArgs {
    const uint64_t* q;
    const uint64_t* r0;
    const uint64_t* r1;
    const double* qinv;  // null: integer products
    uint32_t log_n, limbs;
    size_t total;  // words over all polynomials
};

__device__ __forceinline__ uint64_t mod_product(uint64_t a, uint64_t b, const ElemArgs& e, uint32_t l) {
    const uint64_t q = __ldg(e.q + l);
    if (e.qinv) {
        const DMod md{static_cast<double>(q), __ldg(e.qinv + l)};
        return dto_residue(dmulmod(__ull2double_rn(a), __ull2double_rn(b), md), md);
    }
    return barrett_reduce_128(mul_wide(a, b), q, __ldg(e.r0 + l), __ldg(e.r1 + l));
}

// op 0: a += b, 1: a -= b, 2: a = b - a, 3: a = -a, 4: a *= plain (b is one polynomial)
__global__ void __launch_bounds__(kCkksThreads) k_ckks_elementwise(uint64_t* __restrict__ a,
                                                                  const uint64_t* __restrict__ b, int op,
                                                                  const ElemArgs e) {
    const size_t poly_words = static_cast<size_t>(e.limbs) << e.log_n;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < e.total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t in_poly = i % poly_words;
        const uint32_t l = static_cast<uint32_t>(in_poly >> e.log_n);
        const uint64_t q = __ldg(e.q + l);
        const uint64_t x = a[i];
        uint64_t r;
        switch (op) {
            case 0: r = add_mod(x, b[i], q); break;
            case 1: r = sub_mod(x, b[i], q); break;
            case 2: r = sub_mod(b[i], x, q); break;
            case 3: r = x ? q - x : 0; break;
            default: r = mod_product(x, b[in_poly], e, l); break;
        }
        a[i] = r;
    }
}

// (a0, a1) x (b0, b1) -> (a0 b0, a0 b1 + a1 b0, a1 b1) into a [3][limbs][N]; b may be a
__global__ void __launch_bounds__(kCkksThreads) k_ckks_tensor(uint64_t* a, const uint64_t* b, const ElemArgs e) {
    const size_t poly_words = static_cast<size_t>(e.limbs) << e.log_n;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < poly_words;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t l = static_cast<uint32_t>(i >> e.log_n);
        const uint64_t q = __ldg(e.q + l);
        const uint64_t a0 = a[i], a1 = a[poly_words + i], b0 = b[i], b1 = b[poly_words + i];
        a[i] = mod_product(a0, b0, e, l);
        a[poly_words + i] = add_mod(mod_product(a0, b1, e, l), mod_product(a1, b0, e, l), q);
        a[2 * poly_words + i] = mod_product(a1, b1, e, l);
    }
}

// rescale step 2: tmp[p][j][c] = last[p][c] mod q_j for j < limbs
__global__ void __launch_bounds__(kCkksThreads) k_ckks_last_mod(uint64_t* __restrict__ tmp,
                                                               const uint64_t* __restrict__ last, const ElemArgs e) {
    const size_t n = size_t(1) << e.log_n, poly_words = static_cast<size_t>(e.limbs) << e.log_n;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < e.total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t p = i / poly_words, in_poly = i % poly_words;
        const uint32_t l = static_cast<uint32_t>(in_poly >> e.log_n);
        const uint64_t x = last[p * n + (in_poly & (n - 1))], q = __ldg(e.q + l);
        if (e.qinv) {
            tmp[i] = dto_residue(__ull2double_rn(x), DMod{static_cast<double>(q), __ldg(e.qinv + l)});
        } else {
            tmp[i] = x % q;
        }
    }
}

// dst[l][j] = src[l][perm[j]] (NTT-slot permutation of a Galois automorphism)
__global__ void __launch_bounds__(kCkksThreads) k_ckks_permute(uint64_t* __restrict__ dst,
                                                              const uint64_t* __restrict__ src,
                                                              const uint32_t* __restrict__ perm, uint32_t log_n,
                                                              size_t total) {
    const size_t n = size_t(1) << log_n;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t base = i & ~(n - 1);
        dst[i] = src[base + __ldg(perm + (i & (n - 1)))];
    }
}

unsigned grid_for(size_t total) {
    const size_t b = (total + kCkksThreads - 1) / kCkksThreads;
    return static_cast<unsigned>(b < 148u * 64u ? (b ? b : 1) : 148u * 64u);
}

ElemArgs elem_args(const cbs_rns_context* c, uint32_t limbs, size_t total) {
    return ElemArgs{c->d_q.p, c->d_r0.p, c->d_r1.p, c->d_qinv.p, c->log_n, limbs, total};
}

uint32_t reverse_bits(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

}  // namespace

}  // namespace cbs

using namespace cbs;

extern "C" {

cbs_status cbs_ckks_add_inplace(cbs_rns_context* ctx, uint64_t* d_ct1, const uint64_t* d_ct2, uint32_t size,
                                uint32_t size_ql, cbs_stream_t stream) {
    CBS_CHECK_ARG(d_ct1 && d_ct2, "ckks_add_inplace: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    const size_t total = static_cast<size_t>(size) * size_ql * ctx->n;
    if (!total) return CBS_OK;
    k_ckks_elementwise<<<grid_for(total), kCkksThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        d_ct1, d_ct2, 0, elem_args(ctx, size_ql, total));
    CBS_LAUNCH_CHECK();
    return CBS_OK;
}

cbs_status cbs_ckks_sub_inplace(cbs_rns_context* ctx, uint64_t* d_ct1, const uint64_t* d_ct2, uint32_t size,
                                uint32_t size_ql, int negate, cbs_stream_t stream) {
    CBS_CHECK_ARG(d_ct1 && d_ct2, "ckks_sub_inplace: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    const size_t total = static_cast<size_t>(size) * size_ql * ctx->n;
    if (!total) return CBS_OK;
    k_ckks_elementwise<<<grid_for(total), kCkksThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        d_ct1, d_ct2, negate ? 2 : 1, elem_args(ctx, size_ql, total));
    CBS_LAUNCH_CHECK();
    return CBS_OK;
}

cbs_status cbs_ckks_negate_inplace(cbs_rns_context* ctx, uint64_t* d_ct, uint32_t size, uint32_t size_ql,
                                   cbs_stream_t stream) {
    CBS_CHECK_ARG(d_ct, "ckks_negate_inplace: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    const size_t total = static_cast<size_t>(size) * size_ql * ctx->n;
    if (!total) return CBS_OK;
    k_ckks_elementwise<<<grid_for(total), kCkksThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        d_ct, nullptr, 3, elem_args(ctx, size_ql, total));
    CBS_LAUNCH_CHECK();
    return CBS_OK;
}

cbs_status cbs_ckks_multiply_plain_inplace(cbs_rns_context* ctx, uint64_t* d_ct, const uint64_t* d_plain,
                                           uint32_t size, uint32_t size_ql, cbs_stream_t stream) {
    CBS_CHECK_ARG(d_ct && d_plain, "ckks_multiply_plain_inplace: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    const size_t total = static_cast<size_t>(size) * size_ql * ctx->n;
    if (!total) return CBS_OK;
    k_ckks_elementwise<<<grid_for(total), kCkksThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        d_ct, d_plain, 4, elem_args(ctx, size_ql, total));
    CBS_LAUNCH_CHECK();
    return CBS_OK;
}

cbs_status cbs_ckks_multiply_inplace(cbs_rns_context* ctx, uint64_t* d_ct1, const uint64_t* d_ct2, uint32_t size_ql,
                                     cbs_stream_t stream) {
    CBS_CHECK_ARG(d_ct1 && d_ct2, "ckks_multiply_inplace: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    const size_t words = static_cast<size_t>(size_ql) * ctx->n;
    CBS_CHECK_ARG(d_ct2 == d_ct1 || d_ct2 + 2 * words <= d_ct1 || d_ct1 + 3 * words <= d_ct2,
                  "ckks_multiply_inplace: the operands overlap (pass the same pointer to square)");
    k_ckks_tensor<<<grid_for(words), kCkksThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        d_ct1, d_ct2, elem_args(ctx, size_ql, words));
    CBS_LAUNCH_CHECK();
    return CBS_OK;
}

cbs_status cbs_ckks_relinearize_inplace(cbs_rns_context* ctx, uint64_t* d_ct, const uint64_t* const* h_relin_keys,
                                        uint32_t size_ql, cbs_stream_t stream) {
    CBS_CHECK_ARG(d_ct && h_relin_keys, "ckks_relinearize_inplace: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    const size_t words = static_cast<size_t>(size_ql) * ctx->n;
    return run_keyswitch(ctx, d_ct, d_ct + 2 * words, h_relin_keys, size_ql, 1, static_cast<cudaStream_t>(stream));
}

cbs_status cbs_ckks_multiply_and_relin_inplace(cbs_rns_context* ctx, uint64_t* d_ct1, const uint64_t* d_ct2,
                                               const uint64_t* const* h_relin_keys, uint32_t size_ql,
                                               cbs_stream_t stream) {
    if (cbs_status st = cbs_ckks_multiply_inplace(ctx, d_ct1, d_ct2, size_ql, stream)) return st;
    return cbs_ckks_relinearize_inplace(ctx, d_ct1, h_relin_keys, size_ql, stream);
}

cbs_status cbs_ckks_rescale_to_next(cbs_rns_context* ctx, uint64_t* d_dst, const uint64_t* d_src, uint32_t size,
                                    uint32_t size_ql, cbs_stream_t stream) {
    CBS_CHECK_ARG(d_dst && d_src, "ckks_rescale_to_next: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    CBS_CHECK_ARG(size_ql >= 2, "ckks_rescale_to_next: the ciphertext has no limb to drop");
    if (!size) return CBS_OK;
    cbs_rns_context* c = ctx;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t N = c->n;
    const uint32_t nl = size_ql - 1;
    // q_last^-1 mod q_j and its Shoup form, per level (cached)
    auto it = c->rescale_tab.find(size_ql);
    if (it == c->rescale_tab.end()) {
        std::vector<uint64_t> t(2 * nl);
        const uint64_t qlast = c->primes[nl];
        for (uint32_t j = 0; j < nl; ++j) {
            const uint64_t qj = c->primes[j];
            t[j] = host::invmod(qlast % qj, qj);
            t[nl + j] = host::shoup(t[j], qj);
        }
        auto d = std::make_unique<DevBuf<uint64_t>>();
        CBS_CUDA_TRY(d->upload(t.data(), t.size(), s));
        CBS_CUDA_TRY(cudaStreamSynchronize(s));
        it = c->rescale_tab.emplace(size_ql, std::move(d)).first;
    }
    if (cbs_status st = grow(c->s_ck0, static_cast<size_t>(size) * N)) return st;
    if (cbs_status st = grow(c->s_ck1, static_cast<size_t>(size) * nl * N)) return st;
    // 1. the last limb of every polynomial to the coefficient domain (out of place)
    RnsNttArgs a = c->ntt_args();
    a.limb_prime = c->d_ident.p + nl;  // one launch limb: prime q_last
    a.limbs = 1;
    a.poly_stride = N;
    a.in = d_src + static_cast<size_t>(nl) * N;
    a.in_poly_stride = static_cast<uint64_t>(size_ql) * N;
    CBS_CUDA_TRY(rns_ntt(c->s_ck0.p, a, c->log_n, size, true, s));
    // 2. its residues mod q_0 .. q_{l-1}
    const size_t total = static_cast<size_t>(size) * nl * N;
    k_ckks_last_mod<<<grid_for(total), kCkksThreads, 0, s>>>(c->s_ck1.p, c->s_ck0.p, elem_args(c, nl, total));
    CBS_LAUNCH_CHECK();
    // 3. NTT of those with the epilogue dst = (src_j - v) q_last^-1 (mod q_j)
    RnsNttArgs f = c->ntt_args();
    f.limb_prime = c->d_ident.p;
    f.limbs = nl;
    f.poly_stride = static_cast<uint64_t>(nl) * N;
    f.epi = 1;
    f.epi_cx = d_src;
    f.epi_cx_stride = static_cast<uint64_t>(size_ql) * N;
    f.epi_dst = d_dst;
    f.epi_dst_stride = static_cast<uint64_t>(nl) * N;
    f.epi_f = it->second->p;
    f.epi_fs = it->second->p + nl;
    CBS_CUDA_TRY(rns_ntt(c->s_ck1.p, f, c->log_n, size, false, s));
    return CBS_OK;
}

cbs_status cbs_ckks_mod_switch_to_next(cbs_rns_context* ctx, uint64_t* d_dst, const uint64_t* d_src, uint32_t size,
                                       uint32_t size_ql, cbs_stream_t stream) {
    CBS_CHECK_ARG(d_dst && d_src, "ckks_mod_switch_to_next: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    CBS_CHECK_ARG(size_ql >= 2, "ckks_mod_switch_to_next: the ciphertext has no limb to drop");
    if (!size) return CBS_OK;
    const size_t N = ctx->n, keep = static_cast<size_t>(size_ql - 1) * N * sizeof(uint64_t);
    CBS_CUDA_TRY(cudaMemcpy2DAsync(d_dst, keep, d_src, static_cast<size_t>(size_ql) * N * sizeof(uint64_t), keep, size,
                                   cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
    return CBS_OK;
}

uint32_t cbs_ckks_galois_elt_from_step(int step, uint32_t poly_degree) {
    // rotation by `step` slots: generator 5 raised to step (or to N/2 - |step| for a negative
    // step) mod 2N; step 0 is the conjugation 2N - 1 (include/galois.cuh:17-49)
    const uint32_t n = poly_degree, m = n << 1;
    if (step == 0) return m - 1;
    const uint32_t pos = static_cast<uint32_t>(step < 0 ? -step : step);
    if (n < 2 || pos >= (n >> 1)) return 0;
    uint32_t e = step < 0 ? (n >> 1) - pos : pos;
    uint64_t g = 1;
    while (e--) g = (g * 5u) & (m - 1);
    return static_cast<uint32_t>(g);
}

cbs_status cbs_ckks_apply_galois_inplace(cbs_rns_context* ctx, uint64_t* d_ct, uint32_t galois_elt,
                                         const uint64_t* const* h_galois_keys, uint32_t size_ql, cbs_stream_t stream) {
    CBS_CHECK_ARG(d_ct && h_galois_keys, "ckks_apply_galois_inplace: null argument");
    if (cbs_status st = check_level(ctx, size_ql)) return st;
    cbs_rns_context* c = ctx;
    const uint32_t n = c->n, m = n << 1;
    CBS_CHECK_ARG((galois_elt & 1u) && galois_elt < m, "ckks_apply_galois_inplace: the Galois element must be odd and below 2N");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the NTT-slot permutation of this element (include/galois.cuh:78-91), cached
    auto it = c->galois_perm.find(galois_elt);
    if (it == c->galois_perm.end()) {
        std::vector<uint32_t> perm(n);
        for (uint32_t i = n; i < 2 * n; ++i) {
            const uint32_t rev = reverse_bits(i, static_cast<int>(c->log_n) + 1);
            const uint64_t raw = ((static_cast<uint64_t>(galois_elt) * rev) >> 1) & (n - 1);
            perm[i - n] = reverse_bits(static_cast<uint32_t>(raw), static_cast<int>(c->log_n));
        }
        auto d = std::make_unique<DevBuf<uint32_t>>();
        CBS_CUDA_TRY(d->upload(perm.data(), perm.size(), s));
        CBS_CUDA_TRY(cudaStreamSynchronize(s));
        it = c->galois_perm.emplace(galois_elt, std::move(d)).first;
    }
    const size_t words = static_cast<size_t>(size_ql) * n;
    if (cbs_status st = grow(c->s_ck0, 2 * words)) return st;
    // sigma(c0) back into c0, sigma(c1) kept aside, c1 wiped, then (c0, 0) += KS(sigma(c1))
    k_ckks_permute<<<grid_for(2 * words), kCkksThreads, 0, s>>>(c->s_ck0.p, d_ct, it->second->p, c->log_n, 2 * words);
    CBS_LAUNCH_CHECK();
    CBS_CUDA_TRY(cudaMemcpyAsync(d_ct, c->s_ck0.p, words * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    CBS_CUDA_TRY(cudaMemsetAsync(d_ct + words, 0, words * sizeof(uint64_t), s));
    return run_keyswitch(c, d_ct, c->s_ck0.p + words, h_galois_keys, size_ql, 1, s);
}

cbs_status cbs_ckks_rotate_inplace(cbs_rns_context* ctx, uint64_t* d_ct, int step, const uint64_t* const* h_galois_keys,
                                   uint32_t size_ql, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "ckks_rotate_inplace: null context");
    const uint32_t elt = cbs_ckks_galois_elt_from_step(step, ctx->n);
    CBS_CHECK_ARG(elt != 0, "ckks_rotate_inplace: step count too large");
    return cbs_ckks_apply_galois_inplace(ctx, d_ct, elt, h_galois_keys, size_ql, stream);
}

}  // extern "C"
