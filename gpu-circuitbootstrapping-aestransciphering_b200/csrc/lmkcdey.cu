// lmkcdey.cu -- the LMKCDEY blind rotation (the reference's method = LMKCDEY:
// LMKCDEY_EvalAcc, bitwise/src/cirbts/cirbts-lmkcdey.cu:105-407; its keys,
// cirbts-init.cu:630-726; its place in the bootstrap, cirbts-bootstrap.cu:600-720).
//
// The accumulator is multiplied by RGSW(X^{s_i}) for every LWE coefficient, and the
// coefficients are ordered by the signed base-5 logarithm of their (odd) mask, a_i = +-5^w:
// between groups of equal w the accumulator goes through the automorphism X -> X^{5^k}
// (a key switch from psi(s) back to s), so that after all automorphisms coefficient i has
// contributed X^{a_i s_i}.  The reference runs this one ciphertext at a time from the host,
// ~9 kernel launches per coefficient (INTT, decomposition, NTT, multiply-add, permutations,
// copies) with the bucket order built on the host.
//
// k_lmkcdey: one CTA per ciphertext runs the whole rotation with the accumulator resident
// in shared memory (NTT domain, as the reference keeps it):
//   - the buckets are built in the CTA: every thread maps its masks to buckets through the
//     discrete-log table and counts them with shared atomics, a block scan gives the bucket
//     offsets, and one warp scatters the coefficients stably (index order within a bucket,
//     as the reference's host CSR), so the schedule needs no host round trip;
//   - the walk over the 2 (N/2 - 1) logarithms is uniform across the CTA; per coefficient the
//     external product runs the inverse transforms, the approximate digits (first g-bit
//     digit dropped, as the reference's decomposition) enter the forward transforms on the
//     fly, and the products with the key accumulate in registers (Montgomery form, 64-bit lazy
//     sums); an automorphism gathers the accumulator through its NTT-domain map inside the
//     inverse transform's loads and key-switches the mask component the same way.
// Exact arithmetic mod Q: the accumulator equals the reference's word for word.
#include <cstring>
#include <string>
#include <vector>

#include "cbs_kernels.cuh"
#include "common.cuh"
#include "context.cuh"
#include "ntt_core.cuh"

namespace cbs {

struct LmkArgs {
    RingTables t;
    const uint64_t* a;        // [batch][a_stride] LWE masks mod q_lwe (bootstrap form)
    const uint64_t* b;        // [batch]
    const uint32_t* a_neg;    // [batch][a_stride] negated masks mod 2N (EvalAcc form; null: bootstrap form)
    uint64_t* acc_io;         // EvalAcc form: [batch][2][N] NTT domain, in place
    uint32_t a_stride;
    uint32_t n;
    uint64_t q_lwe;
    uint32_t bitwidth;        // special mod switch of b
    const uint64_t* tv;       // [N] test vector, coefficient domain
    const uint64_t* gadd;     // [num_lut]
    uint32_t num_lut;
    uint64_t* mv_out;         // [batch][num_lut][2][N] NTT domain
    const uint64_t* eval;     // [n][2 digits][2][N] RGSW(X^{s_i}), NTT domain, Montgomery form
    const uint64_t* autok;    // [count][digits][2][N] automorphism keys, NTT domain, Montgomery form
    const uint32_t* maps;     // [count][N] NTT-domain permutations out[t] = in[map[t]]
    const int32_t* log_tab;   // [N] signed base-5 logarithm of the odd residue 2i + 1
    uint32_t num_auto_keys;
    uint32_t window;          // > 1: windowed key set, a skip closes with 5^(q window) then 5^r
    uint32_t digits;
    int gbits;
};

__device__ __forceinline__ int64_t sign_extend(int64_t v, int g) {
    return static_cast<int64_t>(static_cast<uint64_t>(v) << (64 - g)) >> (64 - g);
}

// approximate signed digit d of x (bitwise/src/cirbts/kernel.cu:887-915): the centred value
// in signed g-bit digits from the least significant end, the first digit dropped
__device__ __forceinline__ uint64_t lmk_digit(uint64_t x, uint64_t Q, int g, uint32_t d) {
    int64_t v = x < (Q >> 1) ? static_cast<int64_t>(x) : static_cast<int64_t>(x) - static_cast<int64_t>(Q);
    int64_t r = sign_extend(v, g);
    v = (v - r) >> g;
    for (uint32_t k = 0; k <= d; ++k) {
        r = sign_extend(v, g);
        v = (v - r) >> g;
    }
    return r < 0 ? static_cast<uint64_t>(r + static_cast<int64_t>(Q)) : static_cast<uint64_t>(r);
}

template <int LOGN>
struct LmkCfg {
    static constexpr uint32_t N = 1u << LOGN;
    // acc0, acc1, NTT scratch, coefficient buffer; bucket offsets [N + 1]; items [n]
    static size_t smem(uint32_t n) { return 4ull * N * 8 + (N + 1ull) * 4 + ((2ull * n + 15) / 16) * 16; }
};

template <int LOGN>
__global__ void __launch_bounds__(NttPlan<LOGN>::T, 256 / NttPlan<LOGN>::T + (NttPlan<LOGN>::T < 512))
    k_lmkcdey(const LmkArgs a) {
    constexpr uint32_t N = 1u << LOGN, T = NttPlan<LOGN>::T, TWO_N = 2 * N, NH = N / 2;
    extern __shared__ __align__(16) uint64_t smem[];
    uint64_t* acc0 = smem;
    uint64_t* acc1 = smem + N;
    uint64_t* scr = smem + 2 * N;
    uint64_t* tb = smem + 3 * N;
    uint32_t* offs = reinterpret_cast<uint32_t*>(smem + 4 * N);  // [N + 1] bucket offsets
    uint16_t* items = reinterpret_cast<uint16_t*>(offs + N + 1);  // [n] coefficients by bucket
    __shared__ uint32_t warp_sum[T / 32];
    const uint32_t ct = blockIdx.x, tid = threadIdx.x;
    const RingTables& t = a.t;
    const uint64_t Q = t.q;
    const uint32_t mask = TWO_N - 1, dg = a.digits;
    const int g = a.gbits;
    const bool eval_only = a.a_neg != nullptr;

    // 1. the accumulator: given (EvalAcc form) or (0, X^{-b~} TV) (cirbts-bootstrap.cu:650-674)
    if (eval_only) {
        const uint64_t* in = a.acc_io + static_cast<size_t>(ct) * 2 * N;
        for (uint32_t i = tid; i < 2 * N; i += T) smem[i] = in[i];
    } else {
        const uint32_t bt = special_ms_f(a.b[ct], TWO_N, a.q_lwe, a.bitwidth);
        for (uint32_t i = tid; i < N; i += T) acc0[i] = 0;
        ntt_forward_cta<LOGN>(
            scr, tid, t.rp, t.rps, Q, [&](uint32_t i) { return rot_neg<N>(a.tv, bt, i, Q); },
            [&](int, uint32_t i, uint64_t v) { acc1[i] = v; });
    }
    __syncthreads();

    // 2. buckets (cirbts-lmkcdey.cu:166-214): bucket w + N/2 - 1 for a = 5^w, N/2 - 1 - w for
    //    a = -5^w, N - 1 for a = -1, of the odd residue (-a_neg) | 1
    {
        uint32_t* cnt = reinterpret_cast<uint32_t*>(scr);  // [N] counts, then scatter cursors
        uint32_t* bkt = reinterpret_cast<uint32_t*>(tb);   // [n] bucket of each coefficient
        for (uint32_t i = tid; i < N; i += T) cnt[i] = 0;
        __syncthreads();
        for (uint32_t i = tid; i < a.n; i += T) {
            const size_t at = static_cast<size_t>(ct) * a.a_stride + i;
            const uint32_t an = eval_only ? (__ldg(a.a_neg + at) & mask)
                                          : ((TWO_N - special_ms_f(__ldg(a.a + at), TWO_N, a.q_lwe, 0)) & mask);
            const uint32_t odd = ((0u - an) & mask) | 1u;
            const int32_t lg = __ldg(a.log_tab + (odd >> 1));
            const uint32_t b = lg == static_cast<int32_t>(TWO_N) ? N - 1 : static_cast<uint32_t>(lg + (int32_t)(NH - 1));
            bkt[i] = b;
            atomicAdd(&cnt[b], 1u);
        }
        __syncthreads();
        // exclusive scan: thread tid owns buckets 8 tid .. 8 tid + 7 (T = N / 8)
        uint32_t v[8], run = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            v[j] = run;
            run += cnt[8 * tid + j];
        }
        const uint32_t lane = tid & 31u, warp = tid >> 5;
        uint32_t incl = run;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= static_cast<uint32_t>(d)) incl += o;
        }
        if (lane == 31) warp_sum[warp] = incl;
        __syncthreads();
        uint32_t base = 0;
        for (uint32_t w = 0; w < warp; ++w) base += warp_sum[w];
        base += incl - run;
#pragma unroll
        for (int j = 0; j < 8; ++j) offs[8 * tid + j] = base + v[j];
        if (tid == T - 1) offs[N] = base + run;
        __syncthreads();
        for (uint32_t i = tid; i < N; i += T) cnt[i] = offs[i];
        __syncthreads();
        // stable scatter by one warp: equal buckets keep index order
        if (tid < 32) {
            for (uint32_t b0 = 0; b0 < a.n; b0 += 32) {
                const uint32_t i = b0 + lane;
                const unsigned act = __ballot_sync(0xffffffffu, i < a.n);
                if (i < a.n) {
                    const uint32_t b = bkt[i];
                    const unsigned peers = __match_any_sync(act, b);
                    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
                    items[cnt[b] + rank] = static_cast<uint16_t>(i);
                    __syncwarp(act);
                    if (rank == 0) cnt[b] += __popc(peers);
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }

    // One operation on the accumulator, a single copy of the transform code for both kinds:
    //  - add j: acc <- acc (x) RGSW(X^{s_j}) (AddToAccLMKCDEY_GPU, cirbts-lmkcdey.cu:239-259):
    //    both components' digits against key rows 2d + p;
    //  - automorphism k: acc <- (ks0, psi_k(acc1) + ks1) with ks the key switch of psi_k(acc0)
    //    (AutomorphismLMKCDEY_GPU, cirbts-lmkcdey.cu:261-292); psi_k is a gather through the
    //    NTT-domain map, folded into the inverse transform's loads.
    auto op = [&](bool is_auto, uint32_t arg) {
        const uint32_t* map = a.maps + static_cast<size_t>(is_auto ? arg : 0u) * N;
        const uint64_t* key = is_auto ? a.autok + static_cast<size_t>(arg) * dg * 2 * N
                                      : a.eval + static_cast<size_t>(arg) * 2 * dg * 2 * N;
        const uint32_t polys = is_auto ? 1u : 2u;
        uint64_t s0[8], s1[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) s0[k] = s1[k] = 0;
        for (uint32_t p = 0; p < polys; ++p) {
            const uint64_t* src = p ? acc1 : acc0;
            ntt_inverse_cta<LOGN>(
                scr, tid, t.irp, t.irps, t.n_inv, t.n_inv_s, Q,
                [&](int, uint32_t i) { return is_auto ? acc0[__ldg(map + i)] : src[i]; },
                [&](uint32_t i, uint64_t v) { tb[i] = v; });
            __syncthreads();
            for (uint32_t d = 0; d < dg; ++d) {
                uint64_t x[8];
                ntt_forward_to_regs<LOGN>(
                    scr, tid, t.rp, t.rps, Q, [&](uint32_t i) { return lmk_digit(tb[i], Q, g, d); }, x);
                const uint64_t* k0 = key + static_cast<size_t>(is_auto ? d : 2 * d + p) * 2 * N + 8 * tid;
                const uint64_t* k1 = k0 + N;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    s0[k] += mont_mul_lazy(x[k], __ldg(k0 + k), Q, t.qneg_inv);
                    s1[k] += mont_mul_lazy(x[k], __ldg(k1 + k), Q, t.qneg_inv);
                }
                __syncthreads();
            }
        }
        if (is_auto) {
#pragma unroll
            for (int k = 0; k < 8; ++k) tb[8 * tid + k] = acc1[__ldg(map + 8 * tid + k)];
            __syncthreads();
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t sl = 8 * tid + k;
            acc0[sl] = reduce64(s0[k], Q, t.one_s);
            const uint64_t r1 = reduce64(s1[k], Q, t.one_s);
            acc1[sl] = is_auto ? add_mod(tb[sl], r1, Q) : r1;
        }
        __syncthreads();
    };

    // 3. the walk (cirbts-lmkcdey.cu:322-407): acc1 = psi_{2N-5}(acc1) without key switching
    //    (the mask is zero), then a = -5^w for w = N/2-1 .. 1, a = -1, psi_{2N-5}, a = 5^w for
    //    w = N/2-1 .. 1, a = 1; an automorphism closes every run of w with coefficients and
    //    every num_auto_keys empty steps.  The walk is a generator of operations (uniform
    //    across the CTA), so the operation body is instantiated once.
    {
        uint64_t v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = acc1[__ldg(a.maps + 8 * tid + j)];
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 8; ++j) acc1[8 * tid + j] = v[j];
        __syncthreads();
    }
    uint32_t half = 0, i = NH - 1, pos = 0, hi = 0, skips = 0, stage = 0, pend = 0;
    bool has_pend = false;
    const uint32_t W = a.window;
    // the automorphisms closing a run of sk steps (apply_skip, cirbts-lmkcdey.cu:311-325): the key
    // of 5^sk, or with a window those of 5^(q W) and 5^r (sk = q W + r); the second is left pending
    auto key_of = [W](uint32_t k) { return (W > 1 && k > W) ? W + k / W - 1 : k; };
    auto skip_ops = [&](uint32_t sk, uint32_t& arg) {
        if (W <= 1) {
            arg = sk;
            return;
        }
        const uint32_t q = sk / W, r = sk % W;
        arg = q ? key_of(q * W) : key_of(r);
        if (q && r) {
            pend = key_of(r);
            has_pend = true;
        }
    };
    // the next operation: is_auto and its key (automorphism power index or coefficient)
    auto next = [&](bool& is_auto, uint32_t& arg) -> bool {
        if (has_pend) {
            has_pend = false;
            is_auto = true;
            arg = pend;
            return true;
        }
        for (;;) {
            if (stage == 0) {  // enter the step of logarithm i (i = 0: the special bucket)
                if (i > 0) {
                    const uint32_t b = half == 0 ? (NH - 1) - i : (NH - 1) + i;
                    pos = offs[b];
                    hi = offs[b + 1];
                    stage = 1;
                    if (pos != hi && skips != 0) {
                        is_auto = true;
                        skip_ops(skips, arg);
                        skips = 0;
                        return true;
                    }
                } else {
                    const uint32_t b = half == 0 ? N - 1 : NH - 1;
                    pos = offs[b];
                    hi = offs[b + 1];
                    stage = 3;
                }
            } else if (stage == 1) {  // the step's coefficients, then the skip count
                if (pos < hi) {
                    is_auto = false;
                    arg = items[pos++];
                    return true;
                }
                ++skips;
                stage = 2;
                if ((W <= 1 && skips == a.num_auto_keys) || i == 1) {
                    is_auto = true;
                    skip_ops(skips, arg);
                    skips = 0;
                    return true;
                }
            } else if (stage == 2) {
                --i;
                stage = 0;
            } else {  // the special bucket (a = -1 after the first half, a = 1 after the second)
                if (pos < hi) {
                    is_auto = false;
                    arg = items[pos++];
                    return true;
                }
                if (half == 1) return false;
                half = 1;
                i = NH - 1;
                skips = 0;
                stage = 0;
                is_auto = true;
                arg = 0;
                return true;
            }
        }
    };
    {
        bool is_auto;
        uint32_t arg;
        while (next(is_auto, arg)) op(is_auto, arg);
    }

    if (eval_only) {
        uint64_t* out = a.acc_io + static_cast<size_t>(ct) * 2 * N;
        for (uint32_t i = tid; i < 2 * N; i += T) out[i] = smem[i];
        return;
    }

    // 4. finalize (cirbts-bootstrap.cu:700-717) in the coefficient domain and the MV split
    //    ct_j = acc X^{-j}, emitted in the NTT domain (as the GINX form)
    for (uint32_t p = 0; p < 2; ++p) {
        uint64_t* ap = p ? acc1 : acc0;
        ntt_inverse_cta<LOGN>(
            scr, tid, t.irp, t.irps, t.n_inv, t.n_inv_s, Q, [&](int, uint32_t i) { return ap[i]; },
            [&](uint32_t i, uint64_t v) { ap[i] = v; });
        __syncthreads();
    }
    for (uint32_t i = tid; i < N; i += T) {
        acc0[i] = mul_shoup(acc0[i], t.n_inv, t.n_inv_s, Q);
        uint64_t v = mul_shoup(acc1[i], t.n_inv, t.n_inv_s, Q);
        if (i < a.num_lut) v = add_mod(v, a.gadd[i], Q);
        acc1[i] = v;
    }
    __syncthreads();
    for (uint32_t j = 0; j < a.num_lut; ++j) {
        for (uint32_t p = 0; p < 2; ++p) {
            const uint64_t* src = p ? acc1 : acc0;
            uint64_t* dst = a.mv_out + ((static_cast<size_t>(ct) * a.num_lut + j) * 2 + p) * N;
            ntt_forward_cta<LOGN>(
                scr, tid, t.rp, t.rps, Q, [&](uint32_t i) { return rot_neg<N>(src, j, i, Q); },
                [&](int, uint32_t i, uint64_t v) { dst[i] = v; });
            __syncthreads();
        }
    }
}

template <int LOGN>
static cudaError_t lmk_launch(const LmkArgs& a, uint32_t batch, cudaStream_t s) {
    const size_t smem = LmkCfg<LOGN>::smem(a.n);
    static size_t configured[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (configured[dev] < smem) {
        cudaError_t e =
            cudaFuncSetAttribute(k_lmkcdey<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev] = smem;
    }
    k_lmkcdey<LOGN><<<batch, NttPlan<LOGN>::T, smem, s>>>(a);
    return cudaGetLastError();
}

static cudaError_t launch_lmkcdey(const LmkArgs& a, uint32_t N, uint32_t batch, cudaStream_t s) {
    if (batch == 0) return cudaSuccess;
    switch (N) {
        case 1024: return lmk_launch<10>(a, batch, s);
        case 2048: return lmk_launch<11>(a, batch, s);
        case 4096: return lmk_launch<12>(a, batch, s);
        default: return cudaErrorInvalidValue;
    }
}

// the LMKCDEY keys' generator seed is the key seed xor this constant (context and host agree)
static constexpr uint64_t kLmkSeedTweak = 0x6c6d6b6365797331ull;

// signed base-5 logarithm table of the odd residues of Z_2N (cirbts-lmkcdey.cu:143-176's logGen):
// entry x >> 1 is w for x = 5^w, -w for x = -5^w (w >= 1), 2N for x = -1
static std::vector<int32_t> lmk_log_table(uint32_t N) {
    const uint32_t M = 2 * N;
    std::vector<int32_t> tab(N, 0);
    uint64_t v = 1;
    for (uint32_t w = 0; w < N / 2; ++w) {
        tab[v >> 1] = static_cast<int32_t>(w);
        const uint32_t neg = static_cast<uint32_t>(M - v);
        tab[neg >> 1] = w == 0 ? static_cast<int32_t>(M) : -static_cast<int32_t>(w);
        v = (v * 5) % M;
    }
    return tab;
}

static int bits_of(uint64_t q) {
    int b = 0;
    while (b < 64 && (q >> b)) ++b;
    return b;
}

// the approximate decomposition (first digit dropped) covers Q when g (digits + 1) >= log2 Q
static bool lmk_gadget_ok(const cbs_params& p) {
    int g = 0;
    while ((1u << g) < p.base_g) ++g;
    return g * static_cast<int>(p.digits_g + 1) >= bits_of(p.Q) && g * static_cast<int>(p.digits_g + 1) < 64;
}

static size_t lmk_eval_words(const cbs_params& p) { return static_cast<size_t>(p.n) * 2 * p.digits_g * 2 * p.N; }
static size_t lmk_auto_words(const cbs_params& p, uint32_t num_auto, uint32_t window) {
    return lmkcdey_auto_pows(p.N, num_auto, window).size() * p.digits_g * 2 * p.N;
}

// host keys (c->h_lmk_eval / h_lmk_auto, NTT domain) -> Montgomery-form device keys, maps, log table
static cbs_status upload_lmkcdey(cbs_context* c) {
    FastMod fm(c->p.Q);
    std::vector<uint64_t> ev(c->h_lmk_eval.size()), au(c->h_lmk_auto.size());
    for (size_t i = 0; i < ev.size(); ++i) ev[i] = fm.mul(c->h_lmk_eval[i], c->mont_r);
    for (size_t i = 0; i < au.size(); ++i) au[i] = fm.mul(c->h_lmk_auto[i], c->mont_r);
    std::vector<uint32_t> maps;
    lmkcdey_auto_maps(c->p.N, c->lmk_num_auto, c->lmk_window, maps);
    const auto log_tab = lmk_log_table(c->p.N);
    cudaStream_t s = c->stream;
    CBS_CUDA_TRY(c->d_lmk_eval.upload(ev.data(), ev.size(), s));
    CBS_CUDA_TRY(c->d_lmk_auto.upload(au.data(), au.size(), s));
    CBS_CUDA_TRY(c->d_lmk_maps.upload(maps.data(), maps.size(), s));
    CBS_CUDA_TRY(c->d_lmk_log.upload(log_tab.data(), log_tab.size(), s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    c->lmk_ready = true;
    return CBS_OK;
}

cbs_status prepare_lmkcdey(cbs_context* c) {
    if (c->br_method != CBS_BR_LMKCDEY || c->lmk_ready) return CBS_OK;
    if (!c->keys_ready) return CBS_OK;  // generated with the keys
    if (!c->has_secret) {
        set_error("LMKCDEY blind rotation: generating its keys needs the secret key; "
                  "import them with cbs_import_lmkcdey_keys");
        return CBS_ERR_NOT_READY;
    }
    if (c->device_keyed) {
        set_error("LMKCDEY blind rotation: keys drawn on the device (cbs_keygen_device) have no seeded host "
                  "generator for the LMKCDEY keys; import them with cbs_import_lmkcdey_keys");
        return CBS_ERR_UNSUPPORTED;
    }
    try {
        generate_lmkcdey_keys(c->p, c->tab, c->hk, c->lmk_num_auto, c->lmk_window, c->key_seed ^ kLmkSeedTweak,
                              c->h_lmk_eval,
                              c->h_lmk_auto);
    } catch (const std::exception& e) {
        set_error(std::string("LMKCDEY keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    return upload_lmkcdey(c);
}

static LmkArgs lmk_args(const cbs_context* c) {
    LmkArgs a{};
    a.t = c->ring();
    a.n = c->p.n;
    a.q_lwe = c->p.q_lwe;
    a.bitwidth = c->bitwidth;
    a.tv = c->d_tv.p;
    a.gadd = c->d_gadd.p;
    a.num_lut = c->p.num_lut;
    a.eval = c->d_lmk_eval.p;
    a.autok = c->d_lmk_auto.p;
    a.maps = c->d_lmk_maps.p;
    a.log_tab = c->d_lmk_log.p;
    a.num_auto_keys = c->lmk_num_auto;
    a.window = c->lmk_window > 1 ? c->lmk_window : 0;
    a.digits = c->p.digits_g;
    int g = 0;
    while ((1u << g) < c->p.base_g) ++g;
    a.gbits = g;
    return a;
}

cbs_status run_blind_rotate_lmkcdey(cbs_context* c, const uint64_t* d_a, const uint64_t* d_b, uint32_t batch,
                                    uint32_t a_stride, uint64_t* d_mv, cudaStream_t s) {
    if (!c->lmk_ready) {
        set_error("LMKCDEY blind rotation selected but its keys are not prepared");
        return CBS_ERR_NOT_READY;
    }
    LmkArgs a = lmk_args(c);
    a.a = d_a;
    a.b = d_b;
    a.a_stride = a_stride;
    a.mv_out = d_mv;
    CBS_CUDA_TRY(launch_lmkcdey(a, c->p.N, batch, s));
    return CBS_OK;
}

}  // namespace cbs

using namespace cbs;

extern "C" {

cbs_status cbs_context_set_br_method(cbs_context* ctx, int method, uint32_t num_auto_keys, uint32_t window) {
    CBS_CHECK_ARG(ctx, "set_br_method: null context");
    CBS_CHECK_ARG(method == CBS_BR_GINX || method == CBS_BR_LMKCDEY, "set_br_method: unknown method");
    if (method == CBS_BR_GINX) {
        ctx->br_method = CBS_BR_GINX;
        ctx->aes.drop_graphs();
        return CBS_OK;
    }
    const cbs_params& p = ctx->p;
    CBS_CHECK_ARG(num_auto_keys >= 1 && num_auto_keys < p.N / 2, "set_br_method: num_auto_keys must lie in [1, N/2)");
    CBS_CHECK_ARG(window < p.N / 2, "set_br_method: window must lie in [0, N/2)");
    if (ctx->br_backend != CBS_BR_NTT) {
        set_error("set_br_method: the LMKCDEY blind rotation is implemented for the NTT backend");
        return CBS_ERR_UNSUPPORTED;
    }
    if (!lmk_gadget_ok(p)) {
        set_error("set_br_method: LMKCDEY's approximate decomposition drops one g-bit digit and needs "
                  "g (digits_g + 1) >= log2 Q");
        return CBS_ERR_UNSUPPORTED;
    }
    if (p.num_lut != 1) {
        set_error("set_br_method: LMKCDEY rounds every mask to an odd residue, which a multi-value test vector "
                  "(num_lut > 1, rotations quantized to multiples of 2^bitwidth) cannot absorb; use num_lut = 1");
        return CBS_ERR_UNSUPPORTED;
    }
    CBS_CHECK_ARG(p.n < 65536 && p.n <= 2 * p.N, "set_br_method: LWE dimension too large for the LMKCDEY kernel");
    if (window == 1) window = 0;  // a window of 1 is the plain key set
    if (ctx->br_method != CBS_BR_LMKCDEY || ctx->lmk_num_auto != num_auto_keys || ctx->lmk_window != window) {
        ctx->lmk_ready = false;
        ctx->h_lmk_eval.clear();
        ctx->h_lmk_auto.clear();
    }
    ctx->br_method = CBS_BR_LMKCDEY;
    ctx->lmk_num_auto = num_auto_keys;
    ctx->lmk_window = window;
    ctx->aes.drop_graphs();
    return prepare_lmkcdey(ctx);
}

cbs_status cbs_export_lmkcdey_keys(const cbs_context* ctx, uint64_t* eval, uint64_t* autok, size_t* eval_words,
                                   size_t* auto_words) {
    CBS_CHECK_ARG(ctx && eval_words && auto_words, "export_lmkcdey_keys: null argument");
    if (ctx->br_method != CBS_BR_LMKCDEY || !ctx->lmk_ready) {
        set_error("export_lmkcdey_keys: no LMKCDEY keys (select the method after cbs_keygen)");
        return CBS_ERR_NOT_READY;
    }
    *eval_words = ctx->h_lmk_eval.size();
    *auto_words = ctx->h_lmk_auto.size();
    if (eval) std::memcpy(eval, ctx->h_lmk_eval.data(), ctx->h_lmk_eval.size() * sizeof(uint64_t));
    if (autok) std::memcpy(autok, ctx->h_lmk_auto.data(), ctx->h_lmk_auto.size() * sizeof(uint64_t));
    return CBS_OK;
}

cbs_status cbs_import_lmkcdey_keys(cbs_context* ctx, uint32_t num_auto_keys, uint32_t window, const uint64_t* eval,
                                   size_t eval_words, const uint64_t* autok, size_t auto_words) {
    CBS_CHECK_ARG(ctx && eval && autok, "import_lmkcdey_keys: null argument");
    if (!ctx->keys_ready) {
        set_error("import_lmkcdey_keys: import or generate the keys first");
        return CBS_ERR_NOT_READY;
    }
    const cbs_params& p = ctx->p;
    CBS_CHECK_ARG(num_auto_keys >= 1 && num_auto_keys < p.N / 2 && window < p.N / 2,
                  "import_lmkcdey_keys: num_auto_keys must lie in [1, N/2), window in [0, N/2)");
    if (eval_words != lmk_eval_words(p) || auto_words != lmk_auto_words(p, num_auto_keys, window)) {
        set_error("import_lmkcdey_keys: words must be n * 2 digits_g * 2 N and keys * digits_g * 2 N (keys: 1 + "
                  "num_auto_keys, or with a window 1 + window + floor((N/2 - 1) / window) - 1)");
        return CBS_ERR_SHAPE_MISMATCH;
    }
    for (size_t i = 0; i < eval_words; ++i) CBS_CHECK_ARG(eval[i] < p.Q, "import_lmkcdey_keys: words must be residues");
    for (size_t i = 0; i < auto_words; ++i) CBS_CHECK_ARG(autok[i] < p.Q, "import_lmkcdey_keys: words must be residues");
    // the method's own checks (backend, gadget, num_lut) without generating keys
    const bool had_secret = ctx->has_secret;
    ctx->has_secret = false;
    ctx->br_method = CBS_BR_GINX;
    ctx->lmk_ready = false;
    cbs_status st = cbs_context_set_br_method(ctx, CBS_BR_LMKCDEY, num_auto_keys, window);
    ctx->has_secret = had_secret;
    if (st != CBS_OK && st != CBS_ERR_NOT_READY) {
        ctx->br_method = CBS_BR_GINX;
        return st;
    }
    try {
        ctx->h_lmk_eval.assign(eval, eval + eval_words);
        ctx->h_lmk_auto.assign(autok, autok + auto_words);
    } catch (const std::exception& e) {
        set_error(std::string("import_lmkcdey_keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    return upload_lmkcdey(ctx);
}

cbs_status cbs_generate_lmkcdey_keys_host(const cbs_params* params, uint64_t seed, uint32_t num_auto_keys,
                                          uint32_t window, uint64_t* eval, uint64_t* autok, size_t* eval_words,
                                          size_t* auto_words) {
    CBS_CHECK_ARG(params && eval_words && auto_words, "generate_lmkcdey_keys_host: null argument");
    if (cbs_status st = validate_params(*params)) return st;
    CBS_CHECK_ARG(num_auto_keys >= 1 && num_auto_keys < params->N / 2 && window < params->N / 2,
                  "generate_lmkcdey_keys_host: num_auto_keys must lie in [1, N/2), window in [0, N/2)");
    *eval_words = lmk_eval_words(*params);
    *auto_words = lmk_auto_words(*params, num_auto_keys, window);
    if (!eval || !autok) return CBS_OK;
    host::NttTables t;
    if (!host::make_ntt_tables(params->N, params->Q, t)) {
        set_error("generate_lmkcdey_keys_host: NTT tables failed");
        return CBS_ERR_INVALID_ARG;
    }
    try {
        HostKeys k;
        generate_keys(*params, t, seed, k);
        std::vector<uint64_t> ev, au;
        generate_lmkcdey_keys(*params, t, k, num_auto_keys, window, seed ^ kLmkSeedTweak, ev, au);
        std::memcpy(eval, ev.data(), ev.size() * sizeof(uint64_t));
        std::memcpy(autok, au.data(), au.size() * sizeof(uint64_t));
    } catch (const std::exception& e) {
        set_error(std::string("generate_lmkcdey_keys_host: ") + e.what());
        return CBS_ERR_OOM;
    }
    return CBS_OK;
}

cbs_status cbs_lmkcdey_auto_maps_host(uint32_t N, uint32_t num_auto_keys, uint32_t window, uint32_t* maps,
                                      uint32_t* count) {
    CBS_CHECK_ARG(N >= 64 && (N & (N - 1)) == 0 && num_auto_keys >= 1 && num_auto_keys < N / 2 && window < N / 2,
                  "lmkcdey_auto_maps_host: bad arguments");
    std::vector<uint32_t> m;
    lmkcdey_auto_maps(N, num_auto_keys, window, m);
    if (count) *count = static_cast<uint32_t>(m.size() / N);
    if (!maps) return CBS_OK;
    std::memcpy(maps, m.data(), m.size() * sizeof(uint32_t));
    return CBS_OK;
}

cbs_status cbs_lmkcdey_eval_acc_batch_device(cbs_context* ctx, const uint32_t* d_a_neg, uint32_t a_stride,
                                             uint64_t* d_acc, uint32_t batch, cudaStream_t stream) {
    CBS_CHECK_ARG(ctx && (batch == 0 || (d_a_neg && d_acc)), "lmkcdey_eval_acc: null argument");
    CBS_CHECK_ARG(a_stride >= ctx->p.n, "lmkcdey_eval_acc: a_stride below n");
    if (ctx->br_method != CBS_BR_LMKCDEY || !ctx->lmk_ready) {
        set_error("lmkcdey_eval_acc: select the LMKCDEY method (cbs_context_set_br_method) with its keys first");
        return CBS_ERR_NOT_READY;
    }
    if (batch == 0) return CBS_OK;
    LmkArgs a = lmk_args(ctx);
    a.a_neg = d_a_neg;
    a.acc_io = d_acc;
    a.a_stride = a_stride;
    CBS_CUDA_TRY(launch_lmkcdey(a, ctx->p.N, batch, stream));
    return CBS_OK;
}

}  // extern "C"
