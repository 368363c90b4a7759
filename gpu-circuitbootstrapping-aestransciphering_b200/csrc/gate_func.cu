// gate_func.cu -- functional bootstrapping on the gate context (32-bit torus keys): the
// programmable bootstrap of an LWE ciphertext mod q with an arbitrary test vector
// (BatchGPUBootstrapFunc, bitwise/src/binfhe-base-scheme-batch.cu:215-364) and the evaluators
// built on it (https://eprint.iacr.org/2021/1337, batched as binfhe-base-scheme-batch.cu:366-712):
// EvalFunc, EvalFloor, EvalSign and EvalDecomp.
//
// LWE ciphertexts here are integer vectors mod a power of two 2^bits <= 2^32 (a [count][n],
// b [count], uint32 words), as the reference's LWECiphertext carries its modulus.  The bootstrap
// lifts a ciphertext mod q_in (q_in | 2N) to the torus by a shift, so the blind rotation's
// switch to Z_2N is exact and rotates by multiples of 2N / q_in; the test vector holds
// (2^32 / fmod) f(j) at coefficient j 2N / q_in for j < q_in / 2 (the bootstrap evaluates f on
// [0, q_in / 2) and its negacyclic extension on the other half); the result, key-switched to n,
// is rounded to Z_fmod.  The reference builds the same test vector on the host with b folded in
// and rotates by the masks alone; here b rotates the test vector in the kernel, as the gate
// bootstrap does, so one test vector serves the whole batch.  Every step between bootstraps
// (constant shifts, differences, reductions, modulus switches) is a small element-wise kernel on
// the device: no ciphertext leaves the GPU, where the reference downloads every bootstrap's
// output to finish its key switch on the host.
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "gate_context.cuh"

namespace cbs {

// ciphertexts of one batch: a [count][n] then b [count] (device)
struct LweSet {
    uint32_t* a;
    uint32_t* b;
};

__device__ __forceinline__ uint32_t low_mask(uint32_t bits) { return bits >= 32 ? ~0u : ((1u << bits) - 1u); }

// out = x << shift (a ciphertext mod 2^(32 - shift) on the 32-bit torus)
__global__ void k_lwe_shift(const uint32_t* a, const uint32_t* b, uint32_t* oa, uint32_t* ob, size_t na, uint32_t count,
                            uint32_t shift) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < na + count; i += size_t(gridDim.x) * blockDim.x) {
        if (i < na) oa[i] = a[i] << shift;
        else ob[i - na] = b[i - na] << shift;
    }
}

// x <- floor(0.5 + x 2^to / 2^from) mod 2^to (the reference's RoundqQ, exact for powers of two)
__global__ void k_lwe_round(uint32_t* a, uint32_t* b, size_t na, uint32_t count, uint32_t from_bits, uint32_t to_bits) {
    const uint32_t sh = from_bits - to_bits;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < na + count; i += size_t(gridDim.x) * blockDim.x) {
        uint32_t* p = i < na ? a + i : b + (i - na);
        const uint64_t x = *p;
        const uint64_t r = sh ? (x + (uint64_t(1) << (sh - 1))) >> sh : x;
        *p = static_cast<uint32_t>(r) & low_mask(to_bits);
    }
}

// out = x - y mod 2^bits
__global__ void k_lwe_sub(const uint32_t* xa, const uint32_t* xb, const uint32_t* ya, const uint32_t* yb, uint32_t* oa,
                          uint32_t* ob, size_t na, uint32_t count, uint32_t bits) {
    const uint32_t m = low_mask(bits);
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < na + count; i += size_t(gridDim.x) * blockDim.x) {
        if (i < na) oa[i] = (xa[i] - ya[i]) & m;
        else ob[i - na] = (xb[i - na] - yb[i - na]) & m;
    }
}

// out = x mod 2^bits (the reference's SetModulus to a smaller power of two), b + c first
__global__ void k_lwe_reduce(const uint32_t* a, const uint32_t* b, uint32_t* oa, uint32_t* ob, size_t na,
                             uint32_t count, uint32_t bits, uint32_t add_b) {
    const uint32_t m = low_mask(bits);
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < na + count; i += size_t(gridDim.x) * blockDim.x) {
        if (i < na) oa[i] = a[i] & m;
        else ob[i - na] = (b[i - na] + add_b) & m;
    }
}

namespace {

unsigned elementwise_grid(size_t items) {
    const size_t g = (items + 255) / 256;
    return static_cast<unsigned>(g < 4096 ? (g ? g : 1) : 4096);
}

int pow2_bits(uint64_t v) {
    if (v < 2 || (v & (v - 1))) return -1;
    int b = 0;
    while ((uint64_t(1) << b) < v) ++b;
    return b;
}

struct FuncRun {
    cbs_gate_context* ctx;
    uint32_t count;
    cudaStream_t s;
    size_t na() const { return static_cast<size_t>(count) * ctx->p.n; }

    // the evaluator's k-th scratch set of ciphertexts
    LweSet slot(uint32_t k) const {
        const size_t per = static_cast<size_t>(ctx->max_batch) * (ctx->p.n + 1);
        uint32_t* base = ctx->d_fwork.p + k * per;
        return {base, base + static_cast<size_t>(ctx->max_batch) * ctx->p.n};
    }
    cbs_status shift(LweSet in, LweSet out, uint32_t shift_bits) const {
        k_lwe_shift<<<elementwise_grid(na() + count), 256, 0, s>>>(in.a, in.b, out.a, out.b, na(), count, shift_bits);
        CBS_CUDA_TRY(cudaGetLastError());
        return CBS_OK;
    }
    cbs_status round(LweSet x, uint32_t from_bits, uint32_t to_bits) const {
        k_lwe_round<<<elementwise_grid(na() + count), 256, 0, s>>>(x.a, x.b, na(), count, from_bits, to_bits);
        CBS_CUDA_TRY(cudaGetLastError());
        return CBS_OK;
    }
    cbs_status sub(LweSet x, LweSet y, LweSet out, uint32_t bits) const {
        k_lwe_sub<<<elementwise_grid(na() + count), 256, 0, s>>>(x.a, x.b, y.a, y.b, out.a, out.b, na(), count, bits);
        CBS_CUDA_TRY(cudaGetLastError());
        return CBS_OK;
    }
    // out = (x + (0, c)) mod 2^bits
    cbs_status reduce(LweSet x, LweSet out, uint32_t bits, uint32_t c = 0) const {
        k_lwe_reduce<<<elementwise_grid(na() + count), 256, 0, s>>>(x.a, x.b, out.a, out.b, na(), count, bits, c);
        CBS_CUDA_TRY(cudaGetLastError());
        return CBS_OK;
    }

    // BatchGPUBootstrapFunc: in mod 2^in_bits (in_bits <= log2 2N), f on [0, 2^in_bits / 2)
    // (values mod 2^f_bits) -> out mod 2^f_bits
    cbs_status bootstrap(LweSet in, uint32_t in_bits, const std::vector<uint64_t>& f, uint32_t f_bits, LweSet out) const {
        const cbs_gate_params& p = ctx->p;
        const uint32_t N = p.N, q_in = 1u << in_bits, factor = 2 * N / q_in;
        std::vector<uint32_t> tv(N, 0);
        for (uint32_t j = 0; j < q_in / 2; ++j)
            tv[j * factor] = static_cast<uint32_t>(f[j] << (32 - f_bits));  // (2^32 / fmod) f(j) mod 2^32
        CBS_CUDA_TRY(cudaMemcpyAsync(ctx->d_tv.p, tv.data(), N * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        CBS_CUDA_TRY(cudaStreamSynchronize(s));  // tv is a host temporary
        const LweSet torus{ctx->d_fin_a.p, ctx->d_fin_b.p};
        if (cbs_status st = shift(in, torus, 32 - in_bits)) return st;
        GateArgs a{};
        if (cbs_status st = gate_fill_keys(ctx, a)) return st;
        a.gate = -1;
        a.a1 = torus.a;
        a.b1 = torus.b;
        a.n = p.n;
        a.levels = p.levels;
        a.bg_bits = p.bg_bits;
        a.ext = ctx->d_ext.p;
        a.items = count;
        a.levels_tv = 1;
        a.tv = ctx->d_tv.p;
        CBS_CUDA_TRY(gate_blind_rotate(a, N, count, s));
        CBS_CUDA_TRY(gate_keyswitch(a, ctx->d_ksk.p, p.n, N, p.ks_base_bits, p.ks_levels, out.a, out.b, s));
        return round(out, 32, f_bits);
    }
};

// the reference's checkInputFunction (binfhe-base-scheme.cuh:108-125): 0 negacyclic, 1 periodic, 2 other
uint32_t function_property(const uint32_t* lut, uint64_t q) {
    const uint64_t mid = q / 2;
    if (uint64_t(lut[0]) == q - lut[mid]) {
        for (uint64_t i = 1; i < mid; ++i)
            if (uint64_t(lut[i]) != q - lut[mid + i]) return 2;
        return 0;
    }
    if (lut[0] == lut[mid]) {
        for (uint64_t i = 1; i < mid; ++i)
            if (lut[i] != lut[mid + i]) return 2;
        return 1;
    }
    return 2;
}

// f0 of the reference (binfhe-base-scheme-batch.cu:417-423): -q/4 (as Q - q/4) on the lower half,
// q/4 on the upper half of Z_q; tabulated on [0, q/2) it is the constant Q - q/4
std::vector<uint64_t> half_sign_lut(uint64_t q, uint64_t Q) { return std::vector<uint64_t>(q / 2, Q - (q >> 2)); }

cbs_status prepare(cbs_gate_context* ctx, const void* pa, const void* pb, const void* oa, const void* ob, uint32_t count,
                   const char* who) {
    if (!pa || !pb || !oa || !ob) {
        set_error(std::string(who) + ": null argument");
        return CBS_ERR_INVALID_ARG;
    }
    if (!ctx->keys_ready) {
        set_error(std::string(who) + ": no keys (call cbs_gate_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    if (count > ctx->max_batch) {
        set_error(std::string(who) + ": count above the context's max_batch");
        return CBS_ERR_SHAPE_MISMATCH;
    }
    if (ctx->fft_mode != CBS_FFT_FP64) {
        set_error(std::string(who) + ": functional bootstrapping needs the FP64 external product (cbs_gate_set_fft_mode)");
        return CBS_ERR_UNSUPPORTED;
    }
    const size_t per = static_cast<size_t>(ctx->max_batch) * (ctx->p.n + 1);
    CBS_CUDA_TRY(ctx->d_tv.alloc(ctx->p.N));
    CBS_CUDA_TRY(ctx->d_fin_a.alloc(static_cast<size_t>(ctx->max_batch) * ctx->p.n));
    CBS_CUDA_TRY(ctx->d_fin_b.alloc(ctx->max_batch));
    CBS_CUDA_TRY(ctx->d_fwork.alloc(4 * per));
    return CBS_OK;
}

// EvalFloor on x (mod 2^mod_bits) in place (binfhe-base-scheme-batch.cu:481-543); q = 2^q_bits
cbs_status eval_floor(const FuncRun& r, LweSet x, uint32_t mod_bits, uint32_t q_bits, uint32_t beta) {
    const uint64_t q = uint64_t(1) << q_bits, Q = uint64_t(1) << mod_bits;
    const LweSet ct1 = r.slot(0), low = r.slot(1), ct2 = r.slot(2);
    // ct1 = x + beta; ct2 = bootstrap_f1(ct1 mod q); ct1 -= ct2
    if (cbs_status st = r.reduce(x, ct1, mod_bits, beta)) return st;
    if (cbs_status st = r.reduce(ct1, low, q_bits)) return st;
    if (cbs_status st = r.bootstrap(low, q_bits, half_sign_lut(q, Q), mod_bits, ct2)) return st;
    if (cbs_status st = r.sub(ct1, ct2, ct1, mod_bits)) return st;
    // ct3 = bootstrap_f2(ct1 mod q); x = ct1 - ct3
    std::vector<uint64_t> f2(q / 2);
    for (uint64_t v = 0; v < q / 2; ++v) f2[v] = v < (q >> 2) ? (Q - (q >> 1) - v) & (Q - 1) : v;
    if (cbs_status st = r.reduce(ct1, low, q_bits)) return st;
    if (cbs_status st = r.bootstrap(low, q_bits, f2, mod_bits, ct2)) return st;
    return r.sub(ct1, ct2, x, mod_bits);
}

}  // namespace
}  // namespace cbs

using namespace cbs;

extern "C" {

cbs_status cbs_gate_bootstrap_func_batch_device(cbs_gate_context* ctx, const uint32_t* d_a, const uint32_t* d_b,
                                                uint32_t count, uint32_t q_in, const uint64_t* h_lut, uint64_t fmod,
                                                uint32_t* d_out_a, uint32_t* d_out_b, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && h_lut, "gate_bootstrap_func: null argument");
    const int in_bits = pow2_bits(q_in), f_bits = pow2_bits(fmod);
    CBS_CHECK_ARG(in_bits >= 2 && (1u << in_bits) <= 2 * ctx->p.N, "gate_bootstrap_func: q_in must be a power of two in [4, 2N]");
    CBS_CHECK_ARG(f_bits >= 1 && f_bits <= 32, "gate_bootstrap_func: fmod must be a power of two in [2, 2^32]");
    if (cbs_status st = prepare(ctx, d_a, d_b, d_out_a, d_out_b, count, "gate_bootstrap_func")) return st;
    if (count == 0) return CBS_OK;
    std::vector<uint64_t> f(h_lut, h_lut + q_in / 2);
    for (auto& v : f) CBS_CHECK_ARG(v < fmod, "gate_bootstrap_func: LUT values must lie in [0, fmod)");
    const FuncRun r{ctx, count, reinterpret_cast<cudaStream_t>(stream)};
    return r.bootstrap({const_cast<uint32_t*>(d_a), const_cast<uint32_t*>(d_b)}, in_bits, f, f_bits, {d_out_a, d_out_b});
}

cbs_status cbs_gate_eval_func_batch_device(cbs_gate_context* ctx, const uint32_t* d_a, const uint32_t* d_b,
                                           uint32_t count, uint32_t q, const uint32_t* h_lut, uint32_t beta,
                                           uint32_t* d_out_a, uint32_t* d_out_b, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && h_lut, "gate_eval_func: null argument");
    const int q_bits = pow2_bits(q);
    CBS_CHECK_ARG(q_bits >= 2 && q <= 2 * ctx->p.N, "gate_eval_func: q must be a power of two in [4, 2N]");
    for (uint32_t i = 0; i < q; ++i) CBS_CHECK_ARG(h_lut[i] < q, "gate_eval_func: LUT values must lie in [0, q)");
    if (cbs_status st = prepare(ctx, d_a, d_b, d_out_a, d_out_b, count, "gate_eval_func")) return st;
    const uint32_t prop = function_property(h_lut, q);
    if (prop == 2 && q > ctx->p.N) {
        set_error("gate_eval_func: q must be at most N for an arbitrary (neither negacyclic nor periodic) function");
        return CBS_ERR_INVALID_ARG;
    }
    if (count == 0) return CBS_OK;
    const FuncRun r{ctx, count, reinterpret_cast<cudaStream_t>(stream)};
    const LweSet in{const_cast<uint32_t*>(d_a), const_cast<uint32_t*>(d_b)}, out{d_out_a, d_out_b};
    const LweSet s1 = r.slot(3), s2 = r.slot(2);
    const uint32_t qb = static_cast<uint32_t>(q_bits);
    if (prop == 0) {  // negacyclic: one bootstrap of ct + beta (:382-390)
        if (cbs_status st = r.reduce(in, s1, qb, beta)) return st;
        return r.bootstrap(s1, qb, std::vector<uint64_t>(h_lut, h_lut + q / 2), qb, out);
    }
    if (prop == 2) {  // arbitrary: modulus raised to 2q (:392-449)
        const uint32_t db = qb + 1;
        const uint64_t dq = uint64_t(2) * q;
        if (cbs_status st = r.reduce(in, s1, db, beta)) return st;                 // ct2 = ct1 + beta (mod 2q)
        if (cbs_status st = r.bootstrap(s1, db, half_sign_lut(dq, dq), db, s2)) return st;  // ct3
        if (cbs_status st = r.sub(in, s2, s2, db)) return st;                      // ct3 = ct1 - ct3
        if (cbs_status st = r.reduce(s2, s1, db, beta - (q >> 1))) return st;     // + beta - q/2
        std::vector<uint64_t> f(q);  // fLUT2 on [0, q): LUT2[x] = LUT[x]
        for (uint32_t x = 0; x < q; ++x) f[x] = h_lut[x];
        if (cbs_status st = r.bootstrap(s1, db, f, db, out)) return st;
        return r.reduce(out, out, qb);                                              // SetModulus(q)
    }
    // periodic (:451-477)
    if (cbs_status st = r.reduce(in, s1, qb, beta)) return st;
    if (cbs_status st = r.bootstrap(s1, qb, half_sign_lut(q, q), qb, s2)) return st;  // ct2
    if (cbs_status st = r.sub(in, s2, s2, qb)) return st;                          // ct2 = ct - ct2
    if (cbs_status st = r.reduce(s2, s1, qb, beta - (q >> 2))) return st;         // + beta - q/4
    std::vector<uint64_t> f(q / 2);
    for (uint32_t x = 0; x < q / 2; ++x) f[x] = h_lut[x];  // fLUT1 on [0, q/2)
    return r.bootstrap(s1, qb, f, qb, out);
}

cbs_status cbs_gate_eval_floor_batch_device(cbs_gate_context* ctx, const uint32_t* d_a, const uint32_t* d_b,
                                            uint32_t count, uint64_t mod, uint32_t q, uint32_t roundbits,
                                            uint32_t beta, uint32_t* d_out_a, uint32_t* d_out_b, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "gate_eval_floor: null argument");
    const int mod_bits = pow2_bits(mod);
    const uint64_t qf = roundbits == 0 ? uint64_t(q) : uint64_t(beta) << (roundbits + 1);
    const int q_bits = pow2_bits(qf);
    CBS_CHECK_ARG(mod_bits >= 2 && mod_bits <= 32, "gate_eval_floor: mod must be a power of two in [4, 2^32]");
    CBS_CHECK_ARG(q_bits >= 2 && qf <= 2 * ctx->p.N && q_bits <= mod_bits,
                  "gate_eval_floor: the floor modulus (q, or beta 2^(roundbits+1)) must be a power of two in [4, min(2N, mod)]");
    if (cbs_status st = prepare(ctx, d_a, d_b, d_out_a, d_out_b, count, "gate_eval_floor")) return st;
    if (count == 0) return CBS_OK;
    const FuncRun r{ctx, count, reinterpret_cast<cudaStream_t>(stream)};
    const LweSet x = r.slot(3);
    if (cbs_status st = r.reduce({const_cast<uint32_t*>(d_a), const_cast<uint32_t*>(d_b)}, x, mod_bits)) return st;
    if (cbs_status st = eval_floor(r, x, mod_bits, q_bits, beta)) return st;
    return r.reduce(x, {d_out_a, d_out_b}, mod_bits);
}

cbs_status cbs_gate_eval_sign_batch_device(cbs_gate_context* ctx, const uint32_t* d_a, const uint32_t* d_b,
                                           uint32_t count, uint64_t mod, uint32_t q, uint32_t beta, int scheme_switch,
                                           uint32_t* d_out_a, uint32_t* d_out_b, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "gate_eval_sign: null argument");
    int mod_bits = pow2_bits(mod);
    const int q_bits = pow2_bits(q), beta_bits = pow2_bits(beta);
    CBS_CHECK_ARG(q_bits >= 2 && q <= 2 * ctx->p.N, "gate_eval_sign: q must be a power of two in [4, 2N]");
    CBS_CHECK_ARG(beta_bits >= 1 && beta_bits + 1 < q_bits, "gate_eval_sign: beta must be a power of two below q/2");
    CBS_CHECK_ARG(mod_bits > q_bits && mod_bits <= 32,
                  "gate_eval_sign: for large precision only: mod must be a power of two in (q, 2^32]");
    if (cbs_status st = prepare(ctx, d_a, d_b, d_out_a, d_out_b, count, "gate_eval_sign")) return st;
    if (count == 0) return CBS_OK;
    const FuncRun r{ctx, count, reinterpret_cast<cudaStream_t>(stream)};
    const LweSet x = r.slot(3);
    if (cbs_status st = r.reduce({const_cast<uint32_t*>(d_a), const_cast<uint32_t*>(d_b)}, x, mod_bits)) return st;
    // (binfhe-base-scheme-batch.cu:572-585): floor, then mod <- 2 beta mod / q and switch
    while (mod_bits > q_bits) {
        if (cbs_status st = eval_floor(r, x, mod_bits, q_bits, beta)) return st;
        const int next = mod_bits + 1 + beta_bits - q_bits;
        if (cbs_status st = r.round(x, mod_bits, next)) return st;
        mod_bits = next;
    }
    // the final bootstrap (:608-625): +beta, then Q/4 on the lower half (-Q/4 for scheme switching)
    const LweSet s1 = r.slot(0);
    if (cbs_status st = r.reduce(x, s1, mod_bits, beta)) return st;
    const uint64_t qq = q, half = uint64_t(1) << (mod_bits - 1);
    const std::vector<uint64_t> f3(half, scheme_switch ? qq - qq / 4 : qq / 4);
    if (cbs_status st = r.bootstrap(s1, mod_bits, f3, q_bits, {d_out_a, d_out_b})) return st;
    if (scheme_switch) return CBS_OK;
    return r.reduce({d_out_a, d_out_b}, {d_out_a, d_out_b}, q_bits, 0u - (q >> 2));
}

cbs_status cbs_gate_eval_decomp_batch_device(cbs_gate_context* ctx, const uint32_t* d_a, const uint32_t* d_b,
                                             uint32_t count, uint64_t mod, uint32_t q, uint32_t beta,
                                             uint32_t* d_out_a, uint32_t* d_out_b, uint32_t* digits,
                                             cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && digits, "gate_eval_decomp: null argument");
    int mod_bits = pow2_bits(mod);
    const int q_bits = pow2_bits(q), beta_bits = pow2_bits(beta);
    CBS_CHECK_ARG(q_bits >= 2 && q <= 2 * ctx->p.N, "gate_eval_decomp: q must be a power of two in [4, 2N]");
    CBS_CHECK_ARG(beta_bits >= 1 && beta_bits + 1 < q_bits, "gate_eval_decomp: beta must be a power of two below q/2");
    CBS_CHECK_ARG(mod_bits > q_bits && mod_bits <= 32,
                  "gate_eval_decomp: for large precision only: mod must be a power of two in (q, 2^32]");
    // digits: one per floor (each removes log2(q / 2 beta) bits) and the remainder
    uint32_t need = 1;
    for (int m = mod_bits; m > q_bits; m = m - q_bits + 1 + beta_bits) ++need;
    const uint32_t capacity = *digits;
    *digits = need;
    CBS_CHECK_ARG(capacity >= need, "gate_eval_decomp: the output holds fewer digits than the decomposition makes");
    if (cbs_status st = prepare(ctx, d_a, d_b, d_out_a, d_out_b, count, "gate_eval_decomp")) return st;
    if (count == 0) return CBS_OK;
    const FuncRun r{ctx, count, reinterpret_cast<cudaStream_t>(stream)};
    const LweSet x = r.slot(3);
    if (cbs_status st = r.reduce({const_cast<uint32_t*>(d_a), const_cast<uint32_t*>(d_b)}, x, mod_bits)) return st;
    const size_t na = r.na();
    uint32_t k = 0;
    // (binfhe-base-scheme-batch.cu:656-711): the input mod q is digit k, then floor and switch down
    while (mod_bits > q_bits) {
        if (cbs_status st = r.reduce(x, {d_out_a + k * na, d_out_b + k * size_t(count)}, q_bits)) return st;
        ++k;
        if (cbs_status st = eval_floor(r, x, mod_bits, q_bits, beta)) return st;
        const int next = mod_bits - q_bits + 1 + beta_bits;
        if (cbs_status st = r.round(x, mod_bits, next)) return st;
        mod_bits = next;
    }
    return r.reduce(x, {d_out_a + k * na, d_out_b + k * size_t(count)}, mod_bits);
}

}  // extern "C"
