// rns.cu -- RNS context of the CKKS-style key-switching path: Phantom's 2-D NTT entry points
// and hybrid key switching (modup, key inner product, moddown, keyswitch_inplace).
//
// Follows src/rns_bconv.cu:530-634 (DRNSTool::modup), src/eval_key_switch.cu:13-68
// (key_switch_inner_prod_c2_and_evk), src/rns_bconv.cu:776-828 (DRNSTool::moddown_from_NTT,
// CKKS branch) and src/eval_key_switch.cu:94-181 (keyswitch_inplace, CKKS branch, no level
// dropping beyond the ciphertext's own).  Key modulus chain: the Q primes q_0..q_{L-1}
// followed by the special primes p_0..p_{alpha-1}; digit b of a level-l ciphertext covers
// q_{alpha b} .. q_{min(alpha (b+1), l) - 1}; beta = ceil(l / alpha) digits.
//
// Data layouts (words, uint64 residues, NTT domain unless stated):
//   ciphertext polys  [count][2][Ql][N]           c2        [count][Ql][N]
//   t_mod_up          [count][beta][Ql+P][N]      cx        [count][2][Ql+P][N]
//   evk (per digit b) [2][QP][N]: limb i of the key chain, component 0 then 1
// Results are fully reduced and bit-identical to the reference's kernels: every fast base
// conversion uses the reduced scaled residues [x_i * qhat_i^-1]_{q_i} and an exact 128-bit
// accumulation, so the representation of every intermediate is the reference's.
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "arith.cuh"
#include "common.cuh"
#include "devbuf.cuh"
#include "fp64_mod.cuh"
#include "host_math.h"
#include "ntt_rns.cuh"
#include "rns_context.cuh"

namespace cbs {

constexpr uint32_t kMaxAlpha = 16;   // special primes (= digit width)
constexpr uint32_t kMaxChain = 256;  // primes in Q + P
constexpr uint32_t kMaxBeta = 64;    // digits
constexpr uint32_t kThreads = 256;


struct ModupArgs {
    const uint32_t* out_slot;
    const uint32_t* out_prime;
    const uint64_t* qhat;
    const uint64_t* q;
    const uint64_t* r0;
    const uint64_t* r1;
    uint32_t log_n, ql, qlp, alpha, beta;
    const double* qinv;  // fl(1 / q) per prime, when every prime is below 2^50 (null otherwise)
};

struct EvkPtrs {
    const uint64_t* p[kMaxBeta];
};

struct InnerArgs {
    const uint32_t* prime;  // [qlp] key-chain index
    const uint64_t* q;
    const uint64_t* r0;
    const uint64_t* r1;
    uint32_t log_n, qlp, qp, beta, count, red_k;
};

struct ModdownArgs {
    const uint64_t* phat;
    const uint64_t* q;
    const uint64_t* r0;
    const uint64_t* r1;
    uint32_t log_n, ql, qlp, alpha;
    const double* qinv;  // fl(1 / q) per prime, when every prime is below 2^50 (null otherwise)
};

__device__ __forceinline__ uint64_t barrett(u128 x, const uint64_t* q, const uint64_t* r0, const uint64_t* r1,
                                            uint32_t i) {
    return barrett_reduce_128(x, __ldg(q + i), __ldg(r0 + i), __ldg(r1 + i));
}

// modup, step 2: for digit b = blockIdx.y of ciphertext blockIdx.z, copy the digit's own limbs
// from the NTT-domain input and base-convert its scaled coefficient residues y_i to every
// other limb of Ql+P (src/rns_bconv.cu:455-490 bconv_matmul_padded, :519-527 copy_partQl)
__global__ void __launch_bounds__(kThreads) k_modup_bconv(const uint64_t* __restrict__ coef,
                                                          const uint64_t* __restrict__ c2, uint64_t* __restrict__ t,
                                                          const ModupArgs a) {
    extern __shared__ uint64_t s_qhat[];
    const uint32_t b = blockIdx.y, ct = blockIdx.z;
    const uint32_t start = a.alpha * b;
    const uint32_t cnt = (b == a.beta - 1) ? a.ql - a.alpha * (a.beta - 1) : a.alpha;
    const uint32_t ncompl = a.qlp - cnt;
    const uint64_t* qh = a.qhat + static_cast<size_t>(b) * a.qlp * a.alpha;
    for (uint32_t i = threadIdx.x; i < ncompl * a.alpha; i += blockDim.x) s_qhat[i] = qh[i];
    __syncthreads();
    const size_t N = size_t(1) << a.log_n;
    const size_t c = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t* ci = coef + static_cast<size_t>(ct) * a.ql * N + start * N + c;
    const uint64_t* c2i = c2 + static_cast<size_t>(ct) * a.ql * N + start * N + c;
    uint64_t* tb = t + (static_cast<size_t>(ct) * a.beta + b) * a.qlp * N + c;
    uint64_t y[kMaxAlpha];
#pragma unroll
    for (uint32_t i = 0; i < kMaxAlpha; ++i) {
        if (i < cnt) {
            y[i] = ci[i * N];
            tb[(start + i) * N] = c2i[i * N];
        }
    }
    const uint32_t* slot = a.out_slot + static_cast<size_t>(b) * a.qlp;
    const uint32_t* prime = a.out_prime + static_cast<size_t>(b) * a.qlp;
    for (uint32_t k = 0; k < ncompl; ++k) {
        u128 acc{0, 0};
        const uint64_t* w = s_qhat + k * a.alpha;
#pragma unroll
        for (uint32_t i = 0; i < kMaxAlpha; ++i)
            if (i < cnt) add_wide(acc, mul_wide(y[i], w[i]));
        tb[static_cast<size_t>(__ldg(slot + k)) * N] = barrett(acc, a.q, a.r0, a.r1, __ldg(prime + k));
    }
}

// the same base conversion on the FP64 pipe (every prime below 2^50, fp64_mod.cuh): products
// reduced exactly to |r| <= 0.875 q, partial sums folded every 8 terms; same residues
__global__ void __launch_bounds__(kThreads) k_modup_bconv_d(const uint64_t* __restrict__ coef,
                                                            const uint64_t* __restrict__ c2, uint64_t* __restrict__ t,
                                                            const ModupArgs a) {
    extern __shared__ uint64_t s_qhat[];
    const uint32_t b = blockIdx.y, ct = blockIdx.z;
    const uint32_t start = a.alpha * b;
    const uint32_t cnt = (b == a.beta - 1) ? a.ql - a.alpha * (a.beta - 1) : a.alpha;
    const uint32_t ncompl = a.qlp - cnt;
    const uint64_t* qh = a.qhat + static_cast<size_t>(b) * a.qlp * a.alpha;
    for (uint32_t i = threadIdx.x; i < ncompl * a.alpha; i += blockDim.x) s_qhat[i] = qh[i];
    __syncthreads();
    const size_t N = size_t(1) << a.log_n;
    const size_t c = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t* ci = coef + static_cast<size_t>(ct) * a.ql * N + start * N + c;
    const uint64_t* c2i = c2 + static_cast<size_t>(ct) * a.ql * N + start * N + c;
    uint64_t* tb = t + (static_cast<size_t>(ct) * a.beta + b) * a.qlp * N + c;
    double y[kMaxAlpha];
#pragma unroll
    for (uint32_t i = 0; i < kMaxAlpha; ++i) {
        if (i < cnt) {
            y[i] = __ull2double_rn(ci[i * N]);
            tb[(start + i) * N] = c2i[i * N];
        }
    }
    const uint32_t* slot = a.out_slot + static_cast<size_t>(b) * a.qlp;
    const uint32_t* prime = a.out_prime + static_cast<size_t>(b) * a.qlp;
    for (uint32_t k = 0; k < ncompl; ++k) {
        const uint32_t pk = __ldg(prime + k);
        const DMod md{static_cast<double>(__ldg(a.q + pk)), __ldg(a.qinv + pk)};
        const uint64_t* w = s_qhat + k * a.alpha;
        double acc = 0.0;
#pragma unroll
        for (uint32_t i = 0; i < kMaxAlpha; ++i) {
            if (i < cnt) {
                if (i && (i & 7u) == 0) acc = dreduce(acc, md);
                acc = __dadd_rn(acc, dmulmod(y[i], __ull2double_rn(w[i]), md));
            }
        }
        tb[static_cast<size_t>(__ldg(slot + k)) * N] = dto_residue(acc, md);
    }
}

// key inner product: cx[ct][k][l] = sum_b t[ct][b][l] * evk_b[k][chain(l)] (mod m_l), 128-bit
// accumulation (src/eval_key_switch.cu:13-68).  Each thread covers CT ciphertexts of one
// coefficient so the key words it loads serve CT products.
template <int CT>
__global__ void __launch_bounds__(kThreads) k_ks_inner(const uint64_t* __restrict__ t, const EvkPtrs evk,
                                                       uint64_t* __restrict__ cx, const InnerArgs a) {
    const size_t N = size_t(1) << a.log_n;
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;  // l * N + c
    const uint32_t l = static_cast<uint32_t>(idx >> a.log_n);
    const size_t c = idx & (N - 1);
    const uint32_t pr = __ldg(a.prime + l);
    const uint32_t ct0 = blockIdx.y * CT;
    u128 acc0[CT], acc1[CT];
#pragma unroll
    for (int j = 0; j < CT; ++j) acc0[j] = acc1[j] = u128{0, 0};
    const size_t tstride = static_cast<size_t>(a.beta) * a.qlp * N;  // per ciphertext
    const uint64_t q = __ldg(a.q + pr), r0 = __ldg(a.r0 + pr), r1 = __ldg(a.r1 + pr);
    uint32_t since = 0;
    for (uint32_t b = 0; b < a.beta; ++b) {
        const uint64_t e0 = __ldg(evk.p[b] + static_cast<size_t>(pr) * N + c);
        const uint64_t e1 = __ldg(evk.p[b] + (static_cast<size_t>(a.qp) + pr) * N + c);
        const uint64_t* tb = t + (static_cast<size_t>(b) * a.qlp + l) * N + c;
        if (since == a.red_k) {  // keep the sums below q * 2^64
#pragma unroll
            for (int j = 0; j < CT; ++j) {
                acc0[j] = u128{barrett_reduce_128(acc0[j], q, r0, r1), 0};
                acc1[j] = u128{barrett_reduce_128(acc1[j], q, r0, r1), 0};
            }
            since = 0;
        }
#pragma unroll
        for (int j = 0; j < CT; ++j) {
            if (ct0 + j < a.count) {
                const uint64_t x = tb[(ct0 + j) * tstride];
                add_wide(acc0[j], mul_wide(x, e0));
                add_wide(acc1[j], mul_wide(x, e1));
            }
        }
        ++since;
    }
#pragma unroll
    for (int j = 0; j < CT; ++j) {
        if (ct0 + j < a.count) {
            uint64_t* o = cx + (static_cast<size_t>(ct0 + j) * 2 * a.qlp + l) * N + c;
            o[0] = barrett_reduce_128(acc0[j], q, r0, r1);
            o[static_cast<size_t>(a.qlp) * N] = barrett_reduce_128(acc1[j], q, r0, r1);
        }
    }
}

// the same inner product on the FP64 pipe (every prime below 2^50, fp64_mod.cuh): each product
// is reduced exactly to |r| <= 0.875 q, sums of up to 8 of them are folded back to |x| <= q/2 + 1,
// so every partial sum stays an exact integer below 2^53; same residues as k_ks_inner
template <int CT>
__global__ void __launch_bounds__(kThreads) k_ks_inner_d(const uint64_t* __restrict__ t, const EvkPtrs evk,
                                                         uint64_t* __restrict__ cx, const InnerArgs a) {
    const size_t N = size_t(1) << a.log_n;
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;  // l * N + c
    const uint32_t l = static_cast<uint32_t>(idx >> a.log_n);
    const size_t c = idx & (N - 1);
    const uint32_t pr = __ldg(a.prime + l);
    const uint32_t ct0 = blockIdx.y * CT;
    double acc0[CT], acc1[CT];
#pragma unroll
    for (int j = 0; j < CT; ++j) acc0[j] = acc1[j] = 0.0;
    const size_t tstride = static_cast<size_t>(a.beta) * a.qlp * N;  // per ciphertext
    const DMod md = dmod_of(__ldg(a.q + pr));
    uint32_t since = 0;
    for (uint32_t b = 0; b < a.beta; ++b) {
        const double e0 = __ull2double_rn(__ldg(evk.p[b] + static_cast<size_t>(pr) * N + c));
        const double e1 = __ull2double_rn(__ldg(evk.p[b] + (static_cast<size_t>(a.qp) + pr) * N + c));
        const uint64_t* tb = t + (static_cast<size_t>(b) * a.qlp + l) * N + c;
        if (since == 8) {
#pragma unroll
            for (int j = 0; j < CT; ++j) {
                acc0[j] = dreduce(acc0[j], md);
                acc1[j] = dreduce(acc1[j], md);
            }
            since = 0;
        }
#pragma unroll
        for (int j = 0; j < CT; ++j) {
            if (ct0 + j < a.count) {
                const double x = __ull2double_rn(tb[(ct0 + j) * tstride]);
                acc0[j] = __dadd_rn(acc0[j], dmulmod(x, e0, md));
                acc1[j] = __dadd_rn(acc1[j], dmulmod(x, e1, md));
            }
        }
        ++since;
    }
#pragma unroll
    for (int j = 0; j < CT; ++j) {
        if (ct0 + j < a.count) {
            uint64_t* o = cx + (static_cast<size_t>(ct0 + j) * 2 * a.qlp + l) * N + c;
            o[0] = dto_residue(acc0[j], md);
            o[static_cast<size_t>(a.qlp) * N] = dto_residue(acc1[j], md);
        }
    }
}

// moddown, step 2: delta[poly][i] = sum_j y_j * Phat_j (mod q_i) from the scaled P residues
// (src/rns_bconv.cu:798-801, bConv_BEHZ base_P_to_Ql)
__global__ void __launch_bounds__(kThreads) k_moddown_bconv(const uint64_t* __restrict__ cx,
                                                            uint64_t* __restrict__ delta, const ModdownArgs a) {
    extern __shared__ uint64_t s_phat[];
    for (uint32_t i = threadIdx.x; i < a.ql * a.alpha; i += blockDim.x) s_phat[i] = a.phat[i];
    __syncthreads();
    const size_t N = size_t(1) << a.log_n;
    const size_t c = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t poly = blockIdx.y;
    const uint64_t* src = cx + (static_cast<size_t>(poly) * a.qlp + a.ql) * N + c;
    uint64_t y[kMaxAlpha];
#pragma unroll
    for (uint32_t j = 0; j < kMaxAlpha; ++j)
        if (j < a.alpha) y[j] = src[j * N];
    uint64_t* dst = delta + static_cast<size_t>(poly) * a.ql * N + c;
    for (uint32_t i = 0; i < a.ql; ++i) {
        u128 acc{0, 0};
        const uint64_t* w = s_phat + i * a.alpha;
#pragma unroll
        for (uint32_t j = 0; j < kMaxAlpha; ++j)
            if (j < a.alpha) add_wide(acc, mul_wide(y[j], w[j]));
        dst[i * N] = barrett(acc, a.q, a.r0, a.r1, i);
    }
}

// the same on the FP64 pipe (every prime below 2^50, fp64_mod.cuh); same residues
__global__ void __launch_bounds__(kThreads) k_moddown_bconv_d(const uint64_t* __restrict__ cx,
                                                              uint64_t* __restrict__ delta, const ModdownArgs a) {
    extern __shared__ uint64_t s_phat[];
    for (uint32_t i = threadIdx.x; i < a.ql * a.alpha; i += blockDim.x) s_phat[i] = a.phat[i];
    __syncthreads();
    const size_t N = size_t(1) << a.log_n;
    const size_t c = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t poly = blockIdx.y;
    const uint64_t* src = cx + (static_cast<size_t>(poly) * a.qlp + a.ql) * N + c;
    double y[kMaxAlpha];
#pragma unroll
    for (uint32_t j = 0; j < kMaxAlpha; ++j)
        if (j < a.alpha) y[j] = __ull2double_rn(src[j * N]);
    uint64_t* dst = delta + static_cast<size_t>(poly) * a.ql * N + c;
    for (uint32_t i = 0; i < a.ql; ++i) {
        const DMod md{static_cast<double>(__ldg(a.q + i)), __ldg(a.qinv + i)};
        const uint64_t* w = s_phat + i * a.alpha;
        double acc = 0.0;
#pragma unroll
        for (uint32_t j = 0; j < kMaxAlpha; ++j) {
            if (j < a.alpha) {
                if (j && (j & 7u) == 0) acc = dreduce(acc, md);
                acc = __dadd_rn(acc, dmulmod(y[j], __ull2double_rn(w[j]), md));
            }
        }
        dst[i * N] = dto_residue(acc, md);
    }
}

}  // namespace cbs

using cbs::DevBuf;


namespace {

using cbs::set_error;

template <class T>
cudaError_t upload_sync(DevBuf<T>& b, const std::vector<T>& h) {
    cudaError_t e = b.alloc(h.size());
    if (e != cudaSuccess) return e;
    return cudaMemcpy(b.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

uint64_t prod_mod(const std::vector<uint64_t>& ms, size_t skip, uint64_t m) {
    uint64_t r = 1 % m;
    for (size_t k = 0; k < ms.size(); ++k)
        if (k != skip) r = cbs::host::mulmod(r, ms[k] % m, m);
    return r;
}

}  // namespace

namespace cbs {

// constants of level ql (host restatement of src/rns.cu:120-200 and the BEHZ tables of
// src/rns_base.cu for the part/complement and P/Ql bases)
cbs_status build_level(cbs_rns_context* c, uint32_t ql, cbs::RnsLevel** out) {
    auto it = c->levels.find(ql);
    if (it != c->levels.end()) {
        *out = it->second.get();
        return CBS_OK;
    }
    auto lv = std::make_unique<cbs::RnsLevel>();
    const uint32_t alpha = c->size_p, qlp = ql + alpha, beta = (ql + alpha - 1) / alpha;
    lv->ql = ql;
    lv->qlp = qlp;
    lv->alpha = alpha;
    lv->beta = beta;
    auto chain = [&](uint32_t l) { return l < ql ? l : c->size_q + (l - ql); };  // limb of QlP -> chain
    std::vector<uint64_t> mods(qlp);
    for (uint32_t l = 0; l < qlp; ++l) mods[l] = c->primes[chain(l)];
    // modup
    std::vector<uint64_t> sc(ql), scs(ql), qhat(static_cast<size_t>(beta) * qlp * alpha, 0);
    std::vector<uint32_t> oslot(static_cast<size_t>(beta) * qlp, 0), oprime(static_cast<size_t>(beta) * qlp, 0);
    std::vector<uint32_t> nslot, nprime;
    for (uint32_t b = 0; b < beta; ++b) {
        const uint32_t start = alpha * b, cnt = (b == beta - 1) ? ql - alpha * (beta - 1) : alpha;
        std::vector<uint64_t> part(mods.begin() + start, mods.begin() + start + cnt);
        for (uint32_t i = 0; i < cnt; ++i) {
            const uint64_t qi = part[i];
            sc[start + i] = cbs::host::invmod(prod_mod(part, i, qi), qi);
            scs[start + i] = cbs::host::shoup(sc[start + i], qi);
        }
        uint32_t k = 0;
        for (uint32_t l = 0; l < qlp; ++l) {
            if (l >= start && l < start + cnt) continue;
            oslot[static_cast<size_t>(b) * qlp + k] = l;
            oprime[static_cast<size_t>(b) * qlp + k] = chain(l);
            for (uint32_t i = 0; i < cnt; ++i)
                qhat[(static_cast<size_t>(b) * qlp + k) * alpha + i] = prod_mod(part, i, mods[l]);
            nslot.push_back(b * qlp + l);
            nprime.push_back(chain(l));
            ++k;
        }
    }
    lv->ntt_limbs = static_cast<uint32_t>(nslot.size());
    std::vector<uint32_t> ipr(qlp);
    for (uint32_t l = 0; l < qlp; ++l) ipr[l] = chain(l);
    // moddown
    std::vector<uint64_t> P(c->primes.begin() + c->size_q, c->primes.end());
    std::vector<uint32_t> mslot(alpha), mprime(alpha);
    std::vector<uint64_t> msc(alpha), mscs(alpha), phat(static_cast<size_t>(ql) * alpha), pinv(ql), pinvs(ql);
    for (uint32_t j = 0; j < alpha; ++j) {
        mslot[j] = ql + j;
        mprime[j] = c->size_q + j;
        msc[j] = cbs::host::invmod(prod_mod(P, j, P[j]), P[j]);
        mscs[j] = cbs::host::shoup(msc[j], P[j]);
    }
    for (uint32_t i = 0; i < ql; ++i) {
        const uint64_t qi = c->primes[i];
        for (uint32_t j = 0; j < alpha; ++j) phat[static_cast<size_t>(i) * alpha + j] = prod_mod(P, j, qi);
        pinv[i] = cbs::host::invmod(prod_mod(P, static_cast<size_t>(-1), qi), qi);
        pinvs[i] = cbs::host::shoup(pinv[i], qi);
    }
    CBS_CUDA_TRY(upload_sync(lv->mu_scale, sc));
    CBS_CUDA_TRY(upload_sync(lv->mu_scale_s, scs));
    CBS_CUDA_TRY(upload_sync(lv->mu_out_slot, oslot));
    CBS_CUDA_TRY(upload_sync(lv->mu_out_prime, oprime));
    CBS_CUDA_TRY(upload_sync(lv->mu_qhat, qhat));
    CBS_CUDA_TRY(upload_sync(lv->mu_ntt_slot, nslot));
    CBS_CUDA_TRY(upload_sync(lv->mu_ntt_prime, nprime));
    CBS_CUDA_TRY(upload_sync(lv->ip_prime, ipr));
    CBS_CUDA_TRY(upload_sync(lv->md_slot, mslot));
    CBS_CUDA_TRY(upload_sync(lv->md_prime, mprime));
    CBS_CUDA_TRY(upload_sync(lv->md_scale, msc));
    CBS_CUDA_TRY(upload_sync(lv->md_scale_s, mscs));
    CBS_CUDA_TRY(upload_sync(lv->md_phat, phat));
    CBS_CUDA_TRY(upload_sync(lv->md_pinv, pinv));
    CBS_CUDA_TRY(upload_sync(lv->md_pinv_s, pinvs));
    *out = lv.get();
    c->levels[ql] = std::move(lv);
    return CBS_OK;
}

cbs_status check_level(const cbs_rns_context* c, uint32_t size_ql) {
    CBS_CHECK_ARG(c, "rns: null context");
    CBS_CHECK_ARG(size_ql >= 1 && size_ql <= c->size_q, "rns: size_ql must be in [1, size_q]");
    return CBS_OK;
}

cbs_status grow(DevBuf<uint64_t>& b, size_t words) {
    CBS_CUDA_TRY(b.alloc(words));
    return CBS_OK;
}

}  // namespace cbs

namespace {

using cbs::build_level;
using cbs::check_level;
using cbs::grow;

// modup of count ciphertexts' c2 [count][ql][N] into t [count][beta][qlp][N]
cbs_status run_modup(cbs_rns_context* c, cbs::RnsLevel* lv, uint64_t* d_t, const uint64_t* d_c2, uint32_t count,
                     cudaStream_t s) {
    const size_t N = c->n;
    cbs_status st = grow(c->s_coef, static_cast<size_t>(count) * lv->ql * N);
    if (st != CBS_OK) return st;
    // 1. scaled inverse NTT: coef_i = [INTT(c2_i) * partQlHatInv_i]_{q_i}
    cbs::RnsNttArgs a = c->ntt_args();
    a.limb_prime = c->d_ident.p;
    a.limbs = lv->ql;
    a.poly_stride = static_cast<uint64_t>(lv->ql) * N;
    a.in = d_c2;
    a.in_poly_stride = a.poly_stride;
    a.scale = lv->mu_scale.p;
    a.scale_s = lv->mu_scale_s.p;
    CBS_CUDA_TRY(cbs::rns_ntt(c->s_coef.p, a, c->log_n, count, true, s));
    // 2. base conversion of every digit + copy of its own limbs
    cbs::ModupArgs m{lv->mu_out_slot.p, lv->mu_out_prime.p, lv->mu_qhat.p, c->d_q.p, c->d_r0.p, c->d_r1.p,
                     c->log_n, lv->ql, lv->qlp, lv->alpha, lv->beta};
    const dim3 grid(static_cast<unsigned>(N / cbs::kThreads), lv->beta, count);
    const size_t smem = static_cast<size_t>(lv->qlp) * lv->alpha * sizeof(uint64_t);
    if (c->d_qinv.p) {
        m.qinv = c->d_qinv.p;
        cbs::k_modup_bconv_d<<<grid, cbs::kThreads, smem, s>>>(c->s_coef.p, d_c2, d_t, m);
    } else {
        cbs::k_modup_bconv<<<grid, cbs::kThreads, smem, s>>>(c->s_coef.p, d_c2, d_t, m);
    }
    CBS_LAUNCH_CHECK();
    // 3. forward NTT of every converted limb (the digit's own limbs are already NTT domain)
    cbs::RnsNttArgs f = c->ntt_args();
    f.limb_prime = lv->mu_ntt_prime.p;
    f.limb_slot = lv->mu_ntt_slot.p;
    f.limbs = lv->ntt_limbs;
    f.poly_stride = static_cast<uint64_t>(lv->beta) * lv->qlp * N;
    CBS_CUDA_TRY(cbs::rns_ntt(d_t, f, c->log_n, count, false, s));
    return CBS_OK;
}

cbs_status run_inner(cbs_rns_context* c, cbs::RnsLevel* lv, uint64_t* d_cx, const uint64_t* d_t,
                     const uint64_t* const* h_evks, uint32_t count, cudaStream_t s) {
    cbs::EvkPtrs e{};
    for (uint32_t b = 0; b < lv->beta; ++b) {
        CBS_CHECK_ARG(h_evks[b], "key_switch_inner_prod: null key pointer");
        e.p[b] = h_evks[b];
    }
    constexpr int CT = 4;
    cbs::InnerArgs a{lv->ip_prime.p, c->d_q.p, c->d_r0.p, c->d_r1.p, c->log_n, lv->qlp, c->size_qp,
                     lv->beta, count, c->red_k};
    const dim3 grid(static_cast<unsigned>(static_cast<size_t>(lv->qlp) * c->n / cbs::kThreads), (count + CT - 1) / CT);
    if (c->d_twd.p) cbs::k_ks_inner_d<CT><<<grid, cbs::kThreads, 0, s>>>(d_t, e, d_cx, a);
    else cbs::k_ks_inner<CT><<<grid, cbs::kThreads, 0, s>>>(d_t, e, d_cx, a);
    CBS_LAUNCH_CHECK();
    return CBS_OK;
}

// moddown of polys QlP polys of cx into ct [polys][ql][N]; accumulate adds to ct
cbs_status run_moddown(cbs_rns_context* c, cbs::RnsLevel* lv, uint64_t* d_ct, uint64_t* d_cx, uint32_t polys,
                       bool accumulate, cudaStream_t s) {
    const size_t N = c->n;
    cbs_status st = grow(c->s_delta, static_cast<size_t>(polys) * lv->ql * N);
    if (st != CBS_OK) return st;
    // 1. scaled inverse NTT of the P limbs, in place: y_j = [INTT(cx_Pj) * Phat_j^-1]_{p_j}
    cbs::RnsNttArgs a = c->ntt_args();
    a.limb_prime = lv->md_prime.p;
    a.limb_slot = lv->md_slot.p;
    a.limbs = lv->alpha;
    a.poly_stride = static_cast<uint64_t>(lv->qlp) * N;
    a.scale = lv->md_scale.p;
    a.scale_s = lv->md_scale_s.p;
    CBS_CUDA_TRY(cbs::rns_ntt(d_cx, a, c->log_n, polys, true, s));
    // 2. base conversion P -> Ql
    cbs::ModdownArgs m{lv->md_phat.p, c->d_q.p, c->d_r0.p, c->d_r1.p, c->log_n, lv->ql, lv->qlp, lv->alpha};
    const dim3 grid(static_cast<unsigned>(N / cbs::kThreads), polys);
    const size_t md_smem = static_cast<size_t>(lv->ql) * lv->alpha * sizeof(uint64_t);
    if (c->d_qinv.p) {
        m.qinv = c->d_qinv.p;
        cbs::k_moddown_bconv_d<<<grid, cbs::kThreads, md_smem, s>>>(d_cx, c->s_delta.p, m);
    } else {
        cbs::k_moddown_bconv<<<grid, cbs::kThreads, md_smem, s>>>(d_cx, c->s_delta.p, m);
    }
    CBS_LAUNCH_CHECK();
    // 3. forward NTT of delta with the fused (cx - delta) * P^-1 epilogue
    cbs::RnsNttArgs f = c->ntt_args();
    f.limb_prime = c->d_ident.p;
    f.limbs = lv->ql;
    f.poly_stride = static_cast<uint64_t>(lv->ql) * N;
    f.epi = accumulate ? 2 : 1;
    f.epi_cx = d_cx;
    f.epi_cx_stride = static_cast<uint64_t>(lv->qlp) * N;
    f.epi_dst = d_ct;
    f.epi_dst_stride = static_cast<uint64_t>(lv->ql) * N;
    f.epi_f = lv->md_pinv.p;
    f.epi_fs = lv->md_pinv_s.p;
    CBS_CUDA_TRY(cbs::rns_ntt(c->s_delta.p, f, c->log_n, polys, false, s));
    return CBS_OK;
}

}  // namespace

namespace cbs {

cbs_status run_keyswitch(cbs_rns_context* ctx, uint64_t* d_ct, const uint64_t* d_c2, const uint64_t* const* h_evks,
                         uint32_t size_ql, uint32_t count, cudaStream_t stream) {
    cbs_status st = check_level(ctx, size_ql);
    if (st != CBS_OK) return st;
    CBS_CHECK_ARG(count <= 32767, "rns_keyswitch_inplace: count above 32767");
    if (count == 0) return CBS_OK;
    RnsLevel* lv = nullptr;
    st = build_level(ctx, size_ql, &lv);
    if (st != CBS_OK) return st;
    const size_t N = ctx->n;
    st = grow(ctx->s_t, static_cast<size_t>(count) * lv->beta * lv->qlp * N);
    if (st != CBS_OK) return st;
    st = grow(ctx->s_cx, static_cast<size_t>(count) * 2 * lv->qlp * N);
    if (st != CBS_OK) return st;
    st = run_modup(ctx, lv, ctx->s_t.p, d_c2, count, stream);
    if (st != CBS_OK) return st;
    st = run_inner(ctx, lv, ctx->s_cx.p, ctx->s_t.p, h_evks, count, stream);
    if (st != CBS_OK) return st;
    return run_moddown(ctx, lv, d_ct, ctx->s_cx.p, 2 * count, true, stream);
}

}  // namespace cbs

extern "C" {

cbs_status cbs_rns_context_create(uint32_t poly_degree, const uint64_t* h_q, uint32_t size_q, const uint64_t* h_p,
                                  uint32_t size_p, cbs_rns_context** out) {
    CBS_CHECK_ARG(out && h_q && h_p, "rns_context_create: null argument");
    *out = nullptr;
    const int log_n = cbs::ilog2(poly_degree);
    CBS_CHECK_ARG(poly_degree == (1u << log_n) && log_n >= 10 && log_n <= 17,
                  "rns_context_create: poly_degree must be 2^10 .. 2^17");
    CBS_CHECK_ARG(size_q >= 1 && size_p >= 1 && size_p <= cbs::kMaxAlpha && size_q + size_p <= cbs::kMaxChain,
                  "rns_context_create: need 1 <= size_p <= 16 and size_q + size_p <= 256");
    CBS_CHECK_ARG((size_q + size_p - 1) / size_p <= cbs::kMaxBeta, "rns_context_create: more than 64 digits");
    std::vector<uint64_t> primes(h_q, h_q + size_q);
    primes.insert(primes.end(), h_p, h_p + size_p);
    for (size_t i = 0; i < primes.size(); ++i) {
        const uint64_t q = primes[i];
        CBS_CHECK_ARG(q > 2 && q < (uint64_t(1) << 60) && q % (2ull * poly_degree) == 1 && cbs::host::is_prime(q),
                      "rns_context_create: every modulus must be a prime < 2^60 with q = 1 mod 2N");
        for (size_t k = 0; k < i; ++k) CBS_CHECK_ARG(primes[k] != q, "rns_context_create: duplicate prime");
    }
    auto* c = new (std::nothrow) cbs_rns_context();
    if (!c) {
        set_error("rns_context_create: host allocation failed");
        return CBS_ERR_OOM;
    }
    std::unique_ptr<cbs_rns_context> guard(c);
    c->log_n = static_cast<uint32_t>(log_n);
    c->n = poly_degree;
    c->size_q = size_q;
    c->size_p = size_p;
    c->size_qp = size_q + size_p;
    c->primes = primes;
    CBS_CUDA_TRY(cudaGetDevice(&c->device));
    const size_t N = poly_degree, L = primes.size();
    std::vector<uint64_t> tw(L * N), tws(L * N), itw(L * N), itws(L * N), qv(L), ni(L), nis(L), r0(L), r1(L);
    std::vector<cbs_dmodulus> dm(L);
    std::vector<uint32_t> ident(L);
    uint64_t qmax = 0;
    c->tabs.resize(L);
    for (size_t i = 0; i < L; ++i) {
        auto& t = c->tabs[i];
        if (!cbs::host::make_ntt_tables(poly_degree, primes[i], t)) {
            set_error("rns_context_create: NTT tables failed");
            return CBS_ERR_INVALID_ARG;
        }
        std::copy(t.rp.begin(), t.rp.end(), tw.begin() + i * N);
        std::copy(t.rp_sh.begin(), t.rp_sh.end(), tws.begin() + i * N);
        std::copy(t.irp.begin(), t.irp.end(), itw.begin() + i * N);
        std::copy(t.irp_sh.begin(), t.irp_sh.end(), itws.begin() + i * N);
        qv[i] = primes[i];
        ni[i] = t.n_inv;
        nis[i] = t.n_inv_sh;
        r0[i] = t.ratio0;
        r1[i] = t.ratio1;
        dm[i] = cbs_dmodulus{primes[i], {t.ratio0, t.ratio1}};
        ident[i] = static_cast<uint32_t>(i);
        qmax = std::max(qmax, primes[i]);
    }
    // products added between reductions so that the 128-bit sums stay below q * 2^64
    c->red_k = static_cast<uint32_t>(std::min<uint64_t>(~uint64_t(0) / qmax - 1, 1u << 30));
    if (c->red_k == 0) c->red_k = 1;
    CBS_CUDA_TRY(upload_sync(c->d_tw, tw));
    CBS_CUDA_TRY(upload_sync(c->d_tws, tws));
    CBS_CUDA_TRY(c->d_fault.alloc(1));
    CBS_CUDA_TRY(cudaMemset(c->d_fault.p, 0, sizeof(uint32_t)));
    if (qmax < (uint64_t(1) << 50)) {
        // exact doubles of the twiddles for the FP64-pipe transforms
        std::vector<double> twd(tw.begin(), tw.end()), itwd(itw.begin(), itw.end()), qinv(L);
        for (size_t i = 0; i < L; ++i) qinv[i] = 1.0 / static_cast<double>(primes[i]);
        CBS_CUDA_TRY(upload_sync(c->d_twd, twd));
        CBS_CUDA_TRY(upload_sync(c->d_itwd, itwd));
        CBS_CUDA_TRY(upload_sync(c->d_qinv, qinv));
    }
    CBS_CUDA_TRY(upload_sync(c->d_itw, itw));
    CBS_CUDA_TRY(upload_sync(c->d_itws, itws));
    CBS_CUDA_TRY(upload_sync(c->d_q, qv));
    CBS_CUDA_TRY(upload_sync(c->d_ninv, ni));
    CBS_CUDA_TRY(upload_sync(c->d_ninv_s, nis));
    CBS_CUDA_TRY(upload_sync(c->d_r0, r0));
    CBS_CUDA_TRY(upload_sync(c->d_r1, r1));
    CBS_CUDA_TRY(upload_sync(c->d_mod, dm));
    CBS_CUDA_TRY(upload_sync(c->d_ident, ident));
    *out = guard.release();
    return CBS_OK;
}

cbs_status cbs_rns_context_destroy(cbs_rns_context* ctx) {
    delete ctx;
    return CBS_OK;
}

cbs_status cbs_rns_device_fault(cbs_rns_context* ctx, uint32_t* out, int clear) {
    CBS_CHECK_ARG(ctx && out, "rns_device_fault: null argument");
    CBS_CUDA_TRY(cudaSetDevice(ctx->device));
    CBS_CUDA_TRY(cudaDeviceSynchronize());
    CBS_CUDA_TRY(cudaMemcpy(out, ctx->d_fault.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (clear && *out) CBS_CUDA_TRY(cudaMemset(ctx->d_fault.p, 0, sizeof(uint32_t)));
    return CBS_OK;
}

cbs_status cbs_rns_context_tables(const cbs_rns_context* ctx, cbs_rns_ntt_tables* out) {
    CBS_CHECK_ARG(ctx && out, "rns_context_tables: null argument");
    out->twiddle = ctx->d_tw.p;
    out->twiddle_shoup = ctx->d_tws.p;
    out->itwiddle = ctx->d_itw.p;
    out->itwiddle_shoup = ctx->d_itws.p;
    out->n_inv = ctx->d_ninv.p;
    out->n_inv_shoup = ctx->d_ninv_s.p;
    out->modulus = ctx->d_mod.p;
    out->n = ctx->n;
    out->size = ctx->size_qp;
    return CBS_OK;
}

cbs_status cbs_rns_prepare_level(cbs_rns_context* ctx, uint32_t size_ql) {
    cbs_status st = check_level(ctx, size_ql);
    if (st != CBS_OK) return st;
    cbs::RnsLevel* lv = nullptr;
    return build_level(ctx, size_ql, &lv);
}

cbs_status cbs_rns_ntt_batched(cbs_rns_context* ctx, uint64_t* d_data, uint32_t polys, uint64_t poly_stride,
                               uint32_t coeff_modulus_size, uint32_t start_modulus_idx, int inverse,
                               cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && d_data, "rns_ntt: null argument");
    CBS_CHECK_ARG(coeff_modulus_size >= 1 && start_modulus_idx + coeff_modulus_size <= ctx->size_qp,
                  "rns_ntt: modulus range outside the chain");
    CBS_CHECK_ARG(polys <= 1 || poly_stride >= static_cast<uint64_t>(coeff_modulus_size) * ctx->n,
                  "rns_ntt: poly_stride smaller than one polynomial");
    if (polys == 0) return CBS_OK;
    cbs::RnsNttArgs a = ctx->ntt_args();
    a.limb_prime = ctx->d_ident.p + start_modulus_idx;
    a.limbs = coeff_modulus_size;
    a.poly_stride = poly_stride;
    CBS_CUDA_TRY(cbs::rns_ntt(d_data, a, ctx->log_n, polys, inverse != 0, stream));
    return CBS_OK;
}

cbs_status cbs_nwt_2d_radix8_forward_inplace(cbs_rns_context* ctx, uint64_t* d_inout, uint32_t coeff_modulus_size,
                                             uint32_t start_modulus_idx, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && d_inout, "nwt_2d_radix8_forward_inplace: null argument");
    return cbs_rns_ntt_batched(ctx, d_inout + static_cast<size_t>(start_modulus_idx) * ctx->n, 1, 0,
                               coeff_modulus_size, start_modulus_idx, 0, stream);
}

cbs_status cbs_nwt_2d_radix8_backward_inplace(cbs_rns_context* ctx, uint64_t* d_inout, uint32_t coeff_modulus_size,
                                              uint32_t start_modulus_idx, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && d_inout, "nwt_2d_radix8_backward_inplace: null argument");
    return cbs_rns_ntt_batched(ctx, d_inout + static_cast<size_t>(start_modulus_idx) * ctx->n, 1, 0,
                               coeff_modulus_size, start_modulus_idx, 1, stream);
}

cbs_status cbs_rns_modup(cbs_rns_context* ctx, uint64_t* d_t_mod_up, const uint64_t* d_c2, uint32_t size_ql,
                         uint32_t count, cbs_stream_t stream) {
    cbs_status st = check_level(ctx, size_ql);
    if (st != CBS_OK) return st;
    CBS_CHECK_ARG(d_t_mod_up && d_c2, "rns_modup: null argument");
    CBS_CHECK_ARG(count <= 65535, "rns_modup: count above 65535");
    if (count == 0) return CBS_OK;
    cbs::RnsLevel* lv = nullptr;
    st = build_level(ctx, size_ql, &lv);
    if (st != CBS_OK) return st;
    return run_modup(ctx, lv, d_t_mod_up, d_c2, count, stream);
}

cbs_status cbs_rns_key_switch_inner_prod(cbs_rns_context* ctx, uint64_t* d_cx, const uint64_t* d_t_mod_up,
                                         const uint64_t* const* h_evks, uint32_t size_ql, uint32_t count,
                                         cbs_stream_t stream) {
    cbs_status st = check_level(ctx, size_ql);
    if (st != CBS_OK) return st;
    CBS_CHECK_ARG(d_cx && d_t_mod_up && h_evks, "rns_key_switch_inner_prod: null argument");
    CBS_CHECK_ARG(count <= 65535 * 4, "rns_key_switch_inner_prod: count too large");
    if (count == 0) return CBS_OK;
    cbs::RnsLevel* lv = nullptr;
    st = build_level(ctx, size_ql, &lv);
    if (st != CBS_OK) return st;
    return run_inner(ctx, lv, d_cx, d_t_mod_up, h_evks, count, stream);
}

cbs_status cbs_rns_moddown_from_ntt(cbs_rns_context* ctx, uint64_t* d_ct, uint64_t* d_cx, uint32_t size_ql,
                                    uint32_t polys, int accumulate, cbs_stream_t stream) {
    cbs_status st = check_level(ctx, size_ql);
    if (st != CBS_OK) return st;
    CBS_CHECK_ARG(d_ct && d_cx, "rns_moddown_from_ntt: null argument");
    CBS_CHECK_ARG(polys <= 65535, "rns_moddown_from_ntt: polys above 65535");
    if (polys == 0) return CBS_OK;
    cbs::RnsLevel* lv = nullptr;
    st = build_level(ctx, size_ql, &lv);
    if (st != CBS_OK) return st;
    return run_moddown(ctx, lv, d_ct, d_cx, polys, accumulate != 0, stream);
}

cbs_status cbs_rns_keyswitch_inplace(cbs_rns_context* ctx, uint64_t* d_ct, const uint64_t* d_c2,
                                     const uint64_t* const* h_evks, uint32_t size_ql, uint32_t count,
                                     cbs_stream_t stream) {
    CBS_CHECK_ARG(d_ct && d_c2 && h_evks, "rns_keyswitch_inplace: null argument");
    return cbs::run_keyswitch(ctx, d_ct, d_c2, h_evks, size_ql, count, stream);
}

}  // extern "C"
