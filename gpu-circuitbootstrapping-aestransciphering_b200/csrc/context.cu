// context.cu -- cbs_context lifecycle, key upload, and the batched CBS / CMux / extraction
// entry points of the C ABI.
#include <cstring>
#include <new>
#include <string>

#include "common.cuh"
#include "context.cuh"

namespace cbs {

cudaError_t ntt_forward(uint64_t* out, const uint64_t* in, const uint64_t* tw, const uint64_t* tws,
                        const cbs_dmodulus* mod, size_t dim, size_t batch, cudaStream_t s);
cudaError_t ntt_inverse(uint64_t* out, const uint64_t* in, const uint32_t* map, const uint64_t* itw,
                        const uint64_t* itws, const cbs_dmodulus* mod, const uint64_t* sc, const uint64_t* scs,
                        size_t dim, size_t batch, cudaStream_t s);

static uint64_t neg_inv64(uint64_t q) {
    uint64_t inv = q;  // q * q = 1 mod 8 for odd q
    for (int i = 0; i < 6; ++i) inv *= 2 - q * inv;
    return ~inv + 1;
}

static std::vector<uint64_t> to_mont(const std::vector<uint64_t>& v, const FastMod& fm, uint64_t r) {
    std::vector<uint64_t> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = fm.mul(v[i], r);
    return out;
}

// FFT-domain bootstrapping key and FFT tables for the FP64 backend
static cbs_status prepare_fft(cbs_context* c) {
    if (c->fft_ready) return CBS_OK;
    if (!c->keys_ready) {
        set_error("FFT backend: no key material (call cbs_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    const size_t polys = c->hk.bsk.size() / c->p.N;
    std::vector<double2> bskf, ftab, htf, ssf;
    keys_to_fft_host(c->tab, c->hk.bsk.data(), polys, bskf);
    keys_to_fft_host(c->tab, c->hk.ht.data(), c->hk.ht.size() / c->p.N, htf, kTraceKeySplitBits, 2);
    keys_to_fft_host(c->tab, c->hk.ss.data(), c->hk.ss.size() / c->p.N, ssf, kTraceKeySplitBits, 2);
    fft_tables_host(c->p.N, ftab);
    std::vector<uint64_t> p2(64), p2s(64);
    FastMod fm(c->p.Q);
    uint64_t v = 1 % c->p.Q;
    for (int e = 0; e < 64; ++e) {
        p2[e] = v;
        p2s[e] = host::shoup(v, c->p.Q);
        v = fm.mul(v, 2);
    }
    cudaStream_t s = c->stream;
    CBS_CUDA_TRY(c->d_bskf.upload(bskf.data(), bskf.size(), s));
    CBS_CUDA_TRY(c->d_fft_tab.upload(ftab.data(), ftab.size(), s));
    CBS_CUDA_TRY(c->d_htf.upload(htf.data(), htf.size(), s));
    CBS_CUDA_TRY(c->d_ssf.upload(ssf.data(), ssf.size(), s));
    CBS_CUDA_TRY(c->d_pow2.upload(p2.data(), p2.size(), s));
    CBS_CUDA_TRY(c->d_pow2s.upload(p2s.data(), p2s.size(), s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    c->fft_ready = true;
    return CBS_OK;
}

FftKeyArgs fft_key_args(const cbs_context* c) {
    FftKeyArgs f{};
    f.bskf = c->d_bskf.p;
    f.tab = c->d_fft_tab.p;
    f.tab_len = static_cast<uint32_t>(c->d_fft_tab.n);
    f.pow2 = c->d_pow2.p;
    f.pow2s = c->d_pow2s.p;
    f.inv_m = 2.0 / static_cast<double>(c->p.N);
    f.q_hi = static_cast<double>(c->p.Q);
    f.q_lo = static_cast<double>(static_cast<int64_t>(c->p.Q) - static_cast<int64_t>(f.q_hi));
    f.inv_q = 1.0 / static_cast<double>(c->p.Q);
    return f;
}

static cbs_status make_grouped_keys(cbs_context* c);

// limb spectra of the bootstrapping key (mb = 1) or of the grouped keys (mb = 2, generated here
// unless imported) and the FFT tables for the exact split-FFT backend
static cbs_status prepare_split(cbs_context* c) {
    if (c->split_ready) return CBS_OK;
    if (!c->keys_ready) {
        set_error("split FFT backend: no key material (call cbs_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    const bool grouped = c->br_mb > 1;
    if (grouped && c->h_mbk.empty()) {
        if (cbs_status st = make_grouped_keys(c)) return st;
    }
    const std::vector<uint64_t>& src = grouped ? c->h_mbk : c->hk.bsk;
    const uint32_t per_step = (grouped ? mb_subsets(c->br_mb) : 1u) * 4 * c->p.digits_g;
    std::vector<double2> bskx, ftab;
    try {
        keys_to_fft_limbs_host(c->tab, src.data(), src.size() / c->p.N, per_step, c->split, bskx);
    } catch (const std::exception& e) {
        set_error(std::string("split FFT keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    fft_tables_host(c->p.N, ftab);
    cudaStream_t s = c->stream;
    CBS_CUDA_TRY(c->d_bskx.upload(bskx.data(), bskx.size(), s));
    CBS_CUDA_TRY(c->d_fft_tab.upload(ftab.data(), ftab.size(), s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    c->split_ready = true;
    if (grouped) c->mb_ready = true;
    return CBS_OK;
}

// the limb split of the split-FFT backend for grouping mb, or CBS_ERR_UNSUPPORTED
static cbs_status split_plan_for(const cbs_context* c, uint32_t mb, SplitPlan& plan, const char* who) {
    const int gbits = __builtin_ctz(c->p.base_g);
    if ((c->p.N != 1024 && c->p.N != 2048) || c->p.digits_g < 2 || c->p.digits_g > (mb == 2 ? 3u : 4u) ||
        c->p.base_g > (1u << 24) || !split_plan(c->p.N, c->p.Q, gbits, c->p.digits_g, mb, plan)) {
        set_error(std::string(who) +
                  ": the split FFT backend needs N = 1024 or 2048, 2-4 gadget digits (2-3 for mb = 2) of at most 24 "
                  "bits, mb 1 or 2, and a limb split (at most 4 limbs) whose products stay below 2^50 and Q/2");
        return CBS_ERR_UNSUPPORTED;
    }
    return CBS_OK;
}

static void reset_split(cbs_context* c) {
    c->split_ready = false;
    c->d_bskx.reset();
}

static SplitKeyArgs split_key_args(const cbs_context* c) {
    SplitKeyArgs k{};
    k.bskx = c->d_bskx.p;
    k.limbs = c->split.limbs;
    FastMod fm(c->p.Q);
    const uint64_t base = (uint64_t(1) << c->split.limb_bits) % c->p.Q;  // limb_bits <= 50
    uint64_t v = 1 % c->p.Q;
    for (uint32_t l = 0; l < kMaxSplitLimbs; ++l) {
        k.pw[l] = v;
        k.pws[l] = host::shoup(v, c->p.Q);
        v = fm.mul(v, base);
    }
    return k;
}

// the grouped keys' generator seed is the key seed xor this constant (context and host agree)
static constexpr uint64_t kMbSeedTweak = 0x6d756c7469626974ull;

// grouped multi-bit keys (generated from the context's secrets, seeded from the key seed)
// and their spectra
// spectra of the grouped keys in c->h_mbk, uploaded
static cbs_status upload_mb_spectra(cbs_context* c) {
    std::vector<double2> spec;
    try {
        keys_to_fft_host(c->tab, c->h_mbk.data(), c->h_mbk.size() / c->p.N, spec);
    } catch (const std::exception& e) {
        set_error(std::string("multi-bit keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    CBS_CUDA_TRY(c->d_bskf_mb.upload(spec.data(), spec.size(), c->stream));
    CBS_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->mb_ready = true;
    return CBS_OK;
}

// grouped keys of the context's secrets into c->h_mbk
static cbs_status make_grouped_keys(cbs_context* c) {
    if (!c->keys_ready) {
        set_error("multi-bit blind rotation: no key material (call cbs_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    if (!c->has_secret) {
        set_error("multi-bit blind rotation: generating grouped keys needs the secret key; "
                  "import them with cbs_import_mb_bsk");
        return CBS_ERR_NOT_READY;
    }
    // keys drawn on the device (cbs_keygen_device): the grouped keys from the same stream
    if (c->device_keyed) return device_grouped_keys(c, c->br_mb);
    try {
        generate_mb_bsk(c->p, c->tab, c->hk, c->br_mb, c->key_seed ^ kMbSeedTweak, c->h_mbk);
    } catch (const std::exception& e) {
        set_error(std::string("multi-bit keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    return CBS_OK;
}

static cbs_status prepare_mb(cbs_context* c) {
    if (c->br_mb <= 1 || c->mb_ready) return CBS_OK;
    if (c->br_backend == CBS_BR_FFT64_SPLIT) return prepare_split(c);
    if (cbs_status st = make_grouped_keys(c)) return st;
    return upload_mb_spectra(c);
}

cbs_status apply_tuned_multibit(cbs_context* c) {
    // the cached grouping applies when the caller chose none and the grouped keys can be made
    if (!c->has_tuned || c->mb_explicit || c->tuned.mb == c->br_mb || c->br_backend != CBS_BR_FFT64) return CBS_OK;
    if (c->tuned.mb > 1 && c->keys_ready && !c->has_secret) return CBS_OK;
    c->br_mb = c->tuned.mb;
    c->mb_ready = false;
    c->h_mbk.clear();
    c->d_bskf_mb.reset();
    if (c->br_mb > 1 && c->keys_ready) {
        if (cbs_status st = prepare_mb(c)) return st;
    }
    c->aes.drop_graphs();
    return CBS_OK;
}

cbs_status run_blind_rotate(cbs_context* c, const uint64_t* d_a, const uint64_t* d_b, uint32_t batch,
                            uint32_t a_stride, uint64_t* d_mv, cudaStream_t s, bool mv_ntt) {
    BlindRotateArgs a{};
    a.t = c->ring();
    a.a = d_a;
    a.b = d_b;
    a.a_stride = a_stride;
    a.n = c->p.n;
    a.q_lwe = c->p.q_lwe;
    a.bitwidth = c->bitwidth;
    a.tv = c->d_tv.p;
    a.bsk = c->d_bsk.p;
    a.g = c->g_br;
    a.digits = c->p.digits_g;
    a.num_lut = c->p.num_lut;
    a.gadd = c->d_gadd.p;
    a.mv_out = d_mv;
    a.schedule = c->br_schedule != CBS_BR_SCHEDULE_AUTO ? c->br_schedule
                                                          : (c->has_tuned ? c->tuned.schedule : CBS_BR_SCHEDULE_AUTO);
    if (!mv_ntt && c->br_backend != CBS_BR_FFT64) {
        set_error("coefficient-domain MV output needs the FFT backend");
        return CBS_ERR_INVALID_ARG;
    }
    if (c->br_backend == CBS_BR_FFT64) {
        if (!c->fft_ready) {
            set_error("FFT backend selected but its key material is not prepared");
            return CBS_ERR_NOT_READY;
        }
        if (c->br_mb > 1) {
            if (!c->mb_ready) {
                set_error("multi-bit blind rotation selected but its keys are not prepared");
                return CBS_ERR_NOT_READY;
            }
            FftKeyArgs f = fft_key_args(c);
            f.bskf = c->d_bskf_mb.p;
            CBS_CUDA_TRY(launch_blind_rotate_fft_mb(a, f, c->d_mod.p, c->p.N, batch, c->br_mb, s, mv_ntt));
            return CBS_OK;
        }
        CBS_CUDA_TRY(launch_blind_rotate_fft(a, fft_key_args(c), c->d_mod.p, c->p.N, batch, s, mv_ntt));
        return CBS_OK;
    }
    if (c->br_backend == CBS_BR_FFT64_SPLIT) {
        if (!c->split_ready) {
            set_error("split FFT backend selected but its key material is not prepared");
            return CBS_ERR_NOT_READY;
        }
        CBS_CUDA_TRY(launch_blind_rotate_fft_split(a, fft_key_args(c), split_key_args(c), c->d_mod.p, c->p.N, batch,
                                                   c->br_mb, s));
        return CBS_OK;
    }
    if (c->br_method == CBS_BR_LMKCDEY) return run_blind_rotate_lmkcdey(c, d_a, d_b, batch, a_stride, d_mv, s);
    CBS_CUDA_TRY(launch_blind_rotate(a, c->p.N, batch, s));
    return CBS_OK;
}

cbs_status run_trace(cbs_context* c, const uint64_t* d_mv, uint32_t count, uint64_t* d_rgsw, cudaStream_t s) {
    TraceArgs a{};
    a.t = c->ring();
    a.mv = d_mv;
    a.rgsw = d_rgsw;
    a.maps = c->d_maps.p;
    a.rounds = c->rounds;
    a.ht_key = c->d_ht.p;
    a.ss_key = c->d_ss.p;
    a.g_ht = c->g_ht;
    a.g_ss = c->g_ss;
    a.digits_ht = c->p.digits_ht;
    a.digits_ss = c->p.digits_ss;
    CBS_CUDA_TRY(launch_trace_schemeswitch(a, c->p.N, count, s));
    return CBS_OK;
}

// inverse of the odd k modulo 2^bits (Newton iteration on 2-adic inverses)
static uint32_t inv_pow2(uint32_t k, uint32_t bits) {
    uint32_t x = k;  // k * k = 1 mod 8
    for (int i = 0; i < 5; ++i) x *= 2u - k * x;
    return x & ((bits >= 32) ? ~0u : ((1u << bits) - 1u));
}

cbs_status run_trace_fft(cbs_context* c, const uint64_t* d_mv_coef, uint32_t count, double2* d_rgswf,
                         cudaStream_t s) {
    if (!c->fft_ready) {
        set_error("FFT HomTrace: FFT key material is not prepared");
        return CBS_ERR_NOT_READY;
    }
    TraceFftArgs a{};
    a.mv = d_mv_coef;
    a.rgswf = d_rgswf;
    a.rounds = c->rounds;
    const uint32_t N = c->p.N, logn = static_cast<uint32_t>(__builtin_ctz(N));
    for (uint32_t r = 0; r < c->rounds && r < 16; ++r) a.kinv[r] = inv_pow2((N >> r) + 1, logn + 1);
    a.htf = c->d_htf.p;
    a.ssf = c->d_ssf.p;
    {
        FastMod fm(c->p.Q);
        uint64_t v = 1 % c->p.Q;
        for (uint32_t e = 0; e < kTraceKeySplitBits; ++e) v = fm.mul(v, 2);
        a.split_pow = v;
        a.split_pow_s = host::shoup(v, c->p.Q);
    }
    a.g_ht = make_digit_prep(c->p.Q, c->g_ht, c->p.digits_ht);
    a.g_ss = make_digit_prep(c->p.Q, c->g_ss, c->p.digits_ss);
    a.digits_ht = c->p.digits_ht;
    a.digits_ss = c->p.digits_ss;
    CBS_CUDA_TRY(launch_trace_ss_fft(a, fft_key_args(c), N, count, s));
    return CBS_OK;
}

cbs_status run_cbs(cbs_context* c, const uint64_t* d_a, const uint64_t* d_b, uint32_t batch, uint32_t a_stride,
                   uint64_t* d_mv, uint64_t* d_rgsw, cudaStream_t s) {
    const uint32_t count = batch * c->p.num_lut;
    if (c->br_backend != CBS_BR_FFT64) {
        if (cbs_status st = run_blind_rotate(c, d_a, d_b, batch, a_stride, d_mv, s)) return st;
        return run_trace(c, d_mv, count, d_rgsw, s);
    }
    // FFT backend: coefficient-domain MV RLWEs, FFT HomTrace into row spectra in the output
    // buffer, then back to the NTT-domain reference layout in place
    if (cbs_status st = run_blind_rotate(c, d_a, d_b, batch, a_stride, d_mv, s, false)) return st;
    return run_trace_fft_ntt_rows(c, d_mv, count, d_rgsw, s);
}

cbs_status run_trace_fft_ntt_rows(cbs_context* c, const uint64_t* d_mv_coef, uint32_t count, uint64_t* d_rgsw,
                                  cudaStream_t s) {
    if (cbs_status st = run_trace_fft(c, d_mv_coef, count, reinterpret_cast<double2*>(d_rgsw), s)) return st;
    const size_t polys = static_cast<size_t>(count) * 4;
    CBS_CUDA_TRY(launch_spectra_to_coef(reinterpret_cast<double2*>(d_rgsw), c->p.Q, fft_key_args(c), c->p.N, polys, s));
    CBS_CUDA_TRY(ntt_forward(d_rgsw, d_rgsw, c->d_rp.p, c->d_rps.p, c->d_mod.p, c->p.N, polys, s));
    return CBS_OK;
}

cbs_status build_table_spectra(cbs_context* c, const uint64_t* d_tables, uint64_t table_stride, uint32_t sets,
                               double2* out, cudaStream_t s) {
    CmuxFftArgs a{};
    a.in = d_tables;
    a.in_lut_stride = table_stride;
    a.in_count = 256;
    a.g = make_digit_prep(c->p.Q, c->g_cc, c->p.num_lut);
    a.digits = c->p.num_lut;
    CBS_CUDA_TRY(launch_cmux_pair_spectra(a, fft_key_args(c), c->p.N, sets, out, s));
    return CBS_OK;
}

cbs_status run_lut_levels_fft(cbs_context* c, const uint64_t* d_tables, uint64_t table_stride,
                              const uint32_t* d_lut_sel, const double2* d_rgswf, uint64_t rgsw_stride,
                              const uint32_t* d_ctrl, uint32_t luts, uint64_t* d_buf_a, uint64_t* d_buf_b,
                              uint64_t* d_out, cudaStream_t s, const double2* d_table_spec) {
    const uint32_t N = c->p.N;
    const FftKeyArgs f = fft_key_args(c);
    const uint64_t* in = d_tables;
    for (uint32_t level = 0; level < 8; ++level) {
        CmuxFftArgs a{};
        a.in_count = 256u >> level;
        a.in = in;
        a.in_lut_stride = (level == 0) ? table_stride : static_cast<uint64_t>(a.in_count) * 2 * N;
        a.lut_sel = (level == 0) ? d_lut_sel : nullptr;
        uint64_t* out = (level == 7) ? d_out : ((level & 1) ? d_buf_b : d_buf_a);
        a.out = out;
        a.rgswf = d_rgswf;
        a.rgsw_stride = rgsw_stride;
        a.ctrl_bits = d_ctrl;
        a.level = level;
        a.g = make_digit_prep(c->p.Q, c->g_cc, c->p.num_lut);
        a.digits = c->p.num_lut;
        a.in_spec = (level == 0) ? d_table_spec : nullptr;
        CBS_CUDA_TRY(launch_cmux_level_fft(a, f, N, luts, s));
        in = out;
    }
    return CBS_OK;
}

cbs_status run_lut_levels(cbs_context* c, const uint64_t* d_tables, uint64_t table_stride, const uint32_t* d_lut_sel,
                          const uint64_t* d_rgsw_all, uint64_t rgsw_stride, const uint32_t* d_ctrl, uint32_t luts,
                          uint64_t* d_buf_a, uint64_t* d_buf_b, uint64_t* d_out, cudaStream_t s) {
    const uint32_t N = c->p.N;
    const uint64_t* in = d_tables;
    for (uint32_t level = 0; level < 8; ++level) {
        CmuxLevelArgs a{};
        a.t = c->ring();
        a.in_count = 256u >> level;
        a.in = in;
        a.in_lut_stride = (level == 0) ? table_stride : static_cast<uint64_t>(a.in_count) * 2 * N;
        a.lut_sel = (level == 0) ? d_lut_sel : nullptr;
        uint64_t* out = (level == 7) ? d_out : ((level & 1) ? d_buf_b : d_buf_a);
        a.out = out;
        a.rgsw_all = d_rgsw_all;
        a.rgsw_stride = rgsw_stride;
        a.ctrl_bits = d_ctrl;
        a.level = level;
        a.g = c->g_cc;
        a.digits = c->p.num_lut;
        CBS_CUDA_TRY(launch_cmux_level(a, N, luts, s));
        in = out;
    }
    return CBS_OK;
}

cbs_status run_extract(cbs_context* c, const uint64_t* d_words_coef, const uint32_t* d_info, uint32_t count,
                       uint64_t* d_out_a, uint64_t* d_out_b, uint32_t out_stride, cudaStream_t s) {
    ExtractArgs a{};
    a.words = d_words_coef;
    a.info = d_info;
    a.ksk = c->d_ksk.p;
    a.ksk_stride = ksk_row_stride(c->p.n);
    a.out_a = d_out_a;
    a.out_b = d_out_b;
    a.out_stride = out_stride;
    a.N = c->p.N;
    a.n = c->p.n;
    a.Q = c->p.Q;
    a.q_over_Q = static_cast<double>(c->p.qks) / static_cast<double>(c->p.Q);
    a.qks = c->p.qks;
    a.mask = c->p.qks - 1;
    a.base_ks = c->p.base_ks;
    a.base_log2 = static_cast<uint32_t>(__builtin_ctz(c->p.base_ks));
    a.q_lwe = c->p.q_lwe;
    a.scale = (c->p.q_lwe % c->p.qks == 0) ? c->p.q_lwe / c->p.qks : 0;
    CBS_CUDA_TRY(launch_extract_keyswitch(a, count, s));
    return CBS_OK;
}

static bool pow2(uint64_t x) { return x && !(x & (x - 1)); }

static constexpr double kMaxSigma = 1000.0;

static cbs_status validate(const cbs_params& p) {
    CBS_CHECK_ARG(p.N == 1024 || p.N == 2048 || p.N == 4096, "params: N must be 1024, 2048 or 4096");
    CBS_CHECK_ARG(p.Q > 2 && p.Q < (1ull << 62) && (p.Q - 1) % (2ull * p.N) == 0, "params: Q must be 1 mod 2N, < 2^62");
    CBS_CHECK_ARG(host::is_prime(p.Q), "params: Q must be prime");
    CBS_CHECK_ARG(p.n >= 1 && p.n <= 4096, "params: n out of range");
    CBS_CHECK_ARG(p.q_lwe >= 2 && p.q_lwe <= (1ull << 32), "params: q_lwe out of range");
    CBS_CHECK_ARG(pow2(p.base_g) && p.base_g >= 2 && p.digits_g >= 1 && p.digits_g <= 16, "params: bad BR gadget");
    CBS_CHECK_ARG(p.num_lut >= 1 && p.num_lut <= 8 && pow2(p.base_cc), "params: bad RGSW output gadget");
    CBS_CHECK_ARG(pow2(p.base_ht) && p.digits_ht >= 1 && p.digits_ht <= 16, "params: bad HomTrace gadget");
    CBS_CHECK_ARG(pow2(p.base_ss) && p.digits_ss >= 1 && p.digits_ss <= 16, "params: bad SchemeSwitch gadget");
    CBS_CHECK_ARG(p.trace_shift == 0, "params: only trace_shift = 0 (full HomTrace) is supported");
    CBS_CHECK_ARG(pow2(p.qks) && p.qks <= 65536 && pow2(p.base_ks), "params: qks/base_ks must be powers of two");
    CBS_CHECK_ARG(static_cast<uint64_t>(p.base_ks) * p.base_ks >= p.qks && p.base_ks < p.qks,
                  "params: extraction key switch needs exactly two digits");
    // the discrete-Gaussian samplers tabulate about 14 sigma entries and scan them per sample
    CBS_CHECK_ARG(p.sigma_lwe >= 0 && p.sigma_lwe < kMaxSigma && p.sigma_rlwe >= 0 && p.sigma_rlwe < kMaxSigma,
                  "params: sigma_lwe and sigma_rlwe must lie in [0, 1000)");
    return CBS_OK;
}

cbs_status upload_host_keys(cbs_context* c) {
    FastMod fm(c->p.Q);
    cudaStream_t s = c->stream;
    const auto bsk_m = to_mont(c->hk.bsk, fm, c->mont_r);
    const auto ht_m = to_mont(c->hk.ht, fm, c->mont_r);
    const auto ss_m = to_mont(c->hk.ss, fm, c->mont_r);
    CBS_CUDA_TRY(c->d_bsk.upload(bsk_m.data(), bsk_m.size(), s));
    CBS_CUDA_TRY(c->d_ht.upload(ht_m.data(), ht_m.size(), s));
    CBS_CUDA_TRY(c->d_ss.upload(ss_m.data(), ss_m.size(), s));
    {
        // device copy of the key-switching key with rows padded to ksk_row_stride(n) words
        const size_t rows = c->hk.ksk.size() / (c->p.n + 1), stride = ksk_row_stride(c->p.n);
        std::vector<uint16_t> padded(rows * stride, 0);
        for (size_t r = 0; r < rows; ++r)
            std::memcpy(padded.data() + r * stride, c->hk.ksk.data() + r * (c->p.n + 1),
                        (c->p.n + 1) * sizeof(uint16_t));
        CBS_CUDA_TRY(c->d_ksk.upload(padded.data(), padded.size(), s));
    }
    c->ksk_device_only = false;
    return finish_key_upload(c);
}

cbs_status finish_key_upload(cbs_context* c) {
    cudaStream_t s = c->stream;
    CBS_CUDA_TRY(c->d_tv.upload(c->hk.tv.data(), c->hk.tv.size(), s));
    CBS_CUDA_TRY(c->d_gadd.upload(c->hk.gadd.data(), c->hk.gadd.size(), s));
    CBS_CUDA_TRY(c->d_maps.upload(c->hk.maps.data(), c->hk.maps.size(), s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    c->keys_ready = true;
    c->aes.ready = false;
    c->fft_ready = false;
    c->split_ready = false;
    c->d_bskx.reset();
    c->mb_ready = false;
    c->h_mbk.clear();
    c->d_bskf_mb.reset();
    c->lmk_ready = false;
    c->h_lmk_eval.clear();
    c->h_lmk_auto.clear();
    c->aes.drop_graphs();
    if (c->br_backend == CBS_BR_FFT64) {
        if (cbs_status st = prepare_fft(c)) return st;
        return prepare_mb(c);
    }
    if (c->br_backend == CBS_BR_FFT64_SPLIT) return prepare_split(c);
    // LMKCDEY keys follow from the secrets of a seeded key set (otherwise they are imported)
    if (c->br_method == CBS_BR_LMKCDEY && c->has_secret && !c->device_keyed) return prepare_lmkcdey(c);
    return CBS_OK;
}

cbs_status validate_params(const cbs_params& p) { return validate(p); }

}  // namespace cbs

using namespace cbs;

extern "C" {

cbs_status cbs_params_default(cbs_params* out) {
    CBS_CHECK_ARG(out, "params_default: null output");
    std::vector<uint64_t> q;
    host::get_primes(2048, 54, 1, q);
    cbs_params p{};
    p.N = 2048;
    p.Q = q[0];
    p.n = 630;
    p.q_lwe = 1u << 14;
    p.base_g = 1u << 12;
    p.digits_g = 3;
    p.num_lut = 4;
    p.base_cc = 1u << 6;
    p.base_ht = 1u << 9;
    p.digits_ht = 5;
    p.base_ss = 1u << 9;
    p.digits_ss = 5;
    p.trace_shift = 0;
    p.qks = 1u << 14;
    p.base_ks = 1u << 7;
    p.sigma_lwe = 0.5;
    p.sigma_rlwe = 3.19;
    *out = p;
    return CBS_OK;
}

cbs_status cbs_params_preset(int which, cbs_params* out) {
    CBS_CHECK_ARG(out, "params_preset: null output");
    CBS_CHECK_ARG(which == CBS_PARAMS_AES_3X12 || which == CBS_PARAMS_AES_2X18, "params_preset: unknown preset");
    if (cbs_status st = cbs_params_default(out)) return st;
    if (which == CBS_PARAMS_AES_2X18) {
        out->base_g = 1u << 18;
        out->digits_g = 2;
    }
    return CBS_OK;
}

cbs_status cbs_context_create(const cbs_params* params, uint32_t max_batch, cbs_context** out) {
    CBS_CHECK_ARG(params && out, "context_create: null argument");
    CBS_CHECK_ARG(max_batch >= 1 && max_batch <= (1u << 22), "context_create: max_batch out of range");
    cbs_status st = validate(*params);
    if (st != CBS_OK) return st;
    auto* c = new (std::nothrow) cbs_context();
    if (!c) {
        set_error("context_create: host allocation failed");
        return CBS_ERR_OOM;
    }
    std::unique_ptr<cbs_context> guard(c);
    c->p = *params;
    c->max_batch = max_batch;
    CBS_CUDA_TRY(cudaGetDevice(&c->device));
    if (!host::make_ntt_tables(c->p.N, c->p.Q, c->tab)) {
        set_error("context_create: NTT tables failed");
        return CBS_ERR_INVALID_ARG;
    }
    c->g_br = make_gadget(c->p.Q, c->p.base_g, c->p.digits_g);
    c->g_cc = make_gadget(c->p.Q, c->p.base_cc, c->p.num_lut);
    c->g_ht = make_gadget(c->p.Q, c->p.base_ht, c->p.digits_ht);
    c->g_ss = make_gadget(c->p.Q, c->p.base_ss, c->p.digits_ss);
    c->rounds = static_cast<uint32_t>(__builtin_ctz(c->p.N)) - c->p.trace_shift;
    c->bitwidth = 0;
    while ((1u << c->bitwidth) < c->p.num_lut) ++c->bitwidth;
    c->qneg_inv = neg_inv64(c->p.Q);
    c->one_s = host::shoup(1, c->p.Q);
    c->mont_r = static_cast<uint64_t>((static_cast<unsigned __int128>(1) << 64) % c->p.Q);
    CBS_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const size_t N = c->p.N;
    cudaStream_t s = c->stream;
    CBS_CUDA_TRY(c->d_rp.upload(c->tab.rp.data(), N, s));
    CBS_CUDA_TRY(c->d_rps.upload(c->tab.rp_sh.data(), N, s));
    CBS_CUDA_TRY(c->d_irp.upload(c->tab.irp.data(), N, s));
    CBS_CUDA_TRY(c->d_irps.upload(c->tab.irp_sh.data(), N, s));
    CBS_CUDA_TRY(c->d_ninv.upload(&c->tab.n_inv, 1, s));
    CBS_CUDA_TRY(c->d_ninv_s.upload(&c->tab.n_inv_sh, 1, s));
    cbs_dmodulus dm{c->p.Q, {c->tab.ratio0, c->tab.ratio1}};
    CBS_CUDA_TRY(c->d_mod.upload(&dm, 1, s));
    // scratch for max_batch inputs
    const size_t L = c->p.num_lut;
    CBS_CUDA_TRY(c->d_mv.alloc(static_cast<size_t>(max_batch) * L * 2 * N));
    CBS_CUDA_TRY(c->d_rgsw.alloc(static_cast<size_t>(max_batch) * L * 4 * N));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    c->has_tuned = tune_cache_lookup(c, nullptr, &c->tuned);
    *out = guard.release();
    return CBS_OK;
}

cbs_status cbs_context_destroy(cbs_context* ctx) {
    if (!ctx) return CBS_OK;
    ctx->aes.drop_graphs();
    volatile uint32_t* wipe = ctx->keygen_key.w;  // the key the device key set was drawn with
    for (int i = 0; i < 8; ++i) wipe[i] = 0;
    cudaStream_t s = ctx->stream;
    delete ctx;
    if (s) cudaStreamDestroy(s);
    return CBS_OK;
}

cbs_status cbs_context_stream(const cbs_context* ctx, cbs_stream_t* out) {
    CBS_CHECK_ARG(ctx && out, "context_stream: null argument");
    *out = reinterpret_cast<cbs_stream_t>(ctx->stream);
    return CBS_OK;
}

// upload the evaluation keys of c->hk (bsk / ht / ss to Montgomery form, the KSK with padded
// rows, the derived tables) and rebuild what depends on them

cbs_status cbs_keygen(cbs_context* ctx, uint64_t seed) {
    CBS_CHECK_ARG(ctx, "keygen: null context");
    cbs_context* c = ctx;
    try {
        generate_keys(c->p, c->tab, seed, c->hk);
    } catch (const std::exception& e) {
        set_error(std::string("keygen: ") + e.what());
        return CBS_ERR_OOM;
    }
    c->has_secret = true;
    c->key_seed = seed;
    c->device_keyed = false;
    return upload_host_keys(c);
}

cbs_status cbs_import_keys(cbs_context* ctx, const int32_t* s_lwe, const int32_t* s_rlwe, const uint64_t* bsk,
                           const uint64_t* ht, const uint64_t* ss, const uint16_t* ksk) {
    CBS_CHECK_ARG(ctx && bsk && ht && ss && ksk, "import_keys: null argument (bsk, ht, ss and ksk are required)");
    CBS_CHECK_ARG((s_lwe == nullptr) == (s_rlwe == nullptr), "import_keys: give both secrets or neither");
    cbs_context* c = ctx;
    const cbs_params& p = c->p;
    const uint32_t N = p.N, n = p.n;
    const uint64_t Q = p.Q;
    const size_t n_bsk = static_cast<size_t>(n) * 2 * p.digits_g * 2 * N;
    const size_t n_ht = static_cast<size_t>(c->rounds) * p.digits_ht * 2 * N;
    const size_t n_ss = static_cast<size_t>(p.digits_ss) * 2 * N;
    const size_t n_ksk = static_cast<size_t>(2) * N * p.base_ks * (n + 1);
    auto below_q = [Q](const uint64_t* v, size_t len) {
        for (size_t i = 0; i < len; ++i)
            if (v[i] >= Q) return false;
        return true;
    };
    CBS_CHECK_ARG(below_q(bsk, n_bsk) && below_q(ht, n_ht) && below_q(ss, n_ss),
                  "import_keys: key words must be residues mod Q (NTT domain, the layouts of cbs_export_keys)");
    for (size_t i = 0; i < n_ksk; ++i)
        CBS_CHECK_ARG(ksk[i] < p.qks, "import_keys: key-switching key entries must be below qks");
    if (s_lwe) {
        for (uint32_t i = 0; i < n; ++i)
            CBS_CHECK_ARG(s_lwe[i] == 0 || s_lwe[i] == 1, "import_keys: s_lwe must be binary");
        for (uint32_t i = 0; i < N; ++i)
            CBS_CHECK_ARG(s_rlwe[i] >= -1 && s_rlwe[i] <= 1, "import_keys: s_rlwe must be ternary");
    }
    HostKeys& k = c->hk;
    try {
        k.bsk.assign(bsk, bsk + n_bsk);
        k.ht.assign(ht, ht + n_ht);
        k.ss.assign(ss, ss + n_ss);
        k.ksk.assign(ksk, ksk + n_ksk);
        derive_key_tables(p, k);
        if (s_lwe) {
            set_secrets(p, c->tab, s_lwe, s_rlwe, k);
        } else {
            k.s_lwe.clear();
            k.s_rlwe.clear();
            k.s_ntt.clear();
        }
    } catch (const std::exception& e) {
        set_error(std::string("import_keys: ") + e.what());
        return CBS_ERR_OOM;
    }
    c->has_secret = s_lwe != nullptr;
    c->key_seed = 0;
    return upload_host_keys(c);
}

cbs_status cbs_import_mb_bsk(cbs_context* ctx, uint32_t mb, const uint64_t* keys, size_t words) {
    CBS_CHECK_ARG(ctx && keys, "import_mb_bsk: null argument");
    CBS_CHECK_ARG(mb >= 2 && mb <= 4, "import_mb_bsk: mb must be 2, 3 or 4");
    ctx->mb_explicit = true;
    const bool split = ctx->br_backend == CBS_BR_FFT64_SPLIT;
    if (ctx->br_backend != CBS_BR_FFT64 && !(split && mb == 2)) {
        set_error("import_mb_bsk: grouped blind rotation is implemented for the FFT64 backend (mb 2-4) and the "
                  "split FFT backend (mb 2)");
        return CBS_ERR_UNSUPPORTED;
    }
    SplitPlan plan;
    if (split) {
        if (cbs_status st = split_plan_for(ctx, mb, plan, "import_mb_bsk")) return st;
    }
    if (!ctx->keys_ready) {
        set_error("import_mb_bsk: import or generate the keys first");
        return CBS_ERR_NOT_READY;
    }
    const cbs_params& p = ctx->p;
    const size_t want = static_cast<size_t>((p.n + mb - 1) / mb) * mb_subsets(mb) * 2 * p.digits_g * 2 * p.N;
    if (words != want) {
        set_error("import_mb_bsk: words must be ceil(n/mb) * keys(mb) * 2 digits_g * 2 N (keys 3, 7, 8)");
        return CBS_ERR_SHAPE_MISMATCH;
    }
    for (size_t i = 0; i < words; ++i) CBS_CHECK_ARG(keys[i] < p.Q, "import_mb_bsk: key words must be residues mod Q");
    try {
        ctx->h_mbk.assign(keys, keys + words);
    } catch (const std::exception& e) {
        set_error(std::string("import_mb_bsk: ") + e.what());
        return CBS_ERR_OOM;
    }
    ctx->br_mb = mb;
    ctx->mb_ready = false;
    ctx->aes.drop_graphs();
    if (split) {
        ctx->split = plan;
        reset_split(ctx);
        return prepare_split(ctx);
    }
    return upload_mb_spectra(ctx);
}

cbs_status cbs_context_set_br_schedule(cbs_context* ctx, uint32_t schedule) {
    CBS_CHECK_ARG(ctx, "set_br_schedule: null context");
    CBS_CHECK_ARG(schedule <= CBS_BR_SCHEDULE_PAIRED, "set_br_schedule: unknown schedule");
    ctx->br_schedule = schedule;
    ctx->aes.drop_graphs();  // captured rounds bake in the kernel choice
    return CBS_OK;
}

cbs_status cbs_context_tuned(const cbs_context* ctx, cbs_tune_choice* out) {
    CBS_CHECK_ARG(ctx && out, "context_tuned: null argument");
    if (!ctx->has_tuned) {
        set_error("context_tuned: no tuning-cache entry for this GPU and parameter set");
        return CBS_ERR_NOT_READY;
    }
    *out = ctx->tuned;
    return CBS_OK;
}

cbs_status cbs_context_set_br_multibit(cbs_context* ctx, uint32_t mb) {
    CBS_CHECK_ARG(ctx, "set_br_multibit: null context");
    CBS_CHECK_ARG(mb >= 1 && mb <= 4, "set_br_multibit: mb must be 1, 2, 3 or 4");
    ctx->mb_explicit = true;
    const bool split = ctx->br_backend == CBS_BR_FFT64_SPLIT;
    if (mb > 1 && ctx->br_backend != CBS_BR_FFT64 && !(split && mb == 2)) {
        set_error("set_br_multibit: grouped blind rotation is implemented for the FFT64 backend (mb 2-4) and the "
                  "split FFT backend (mb 2)");
        return CBS_ERR_UNSUPPORTED;
    }
    SplitPlan plan;
    if (split) {
        if (cbs_status st = split_plan_for(ctx, mb, plan, "set_br_multibit")) return st;
    }
    if (mb != ctx->br_mb) {
        ctx->br_mb = mb;
        ctx->mb_ready = false;
        ctx->h_mbk.clear();
        ctx->d_bskf_mb.reset();
        reset_split(ctx);
    }
    if (split) ctx->split = plan;
    if (split && ctx->keys_ready) {  // limb spectra of the BSK (mb = 1) or of the grouped keys
        if (cbs_status st = prepare_split(ctx)) return st;
    } else if (mb > 1 && ctx->keys_ready) {
        if (cbs_status st = prepare_mb(ctx)) return st;
    }
    ctx->aes.drop_graphs();
    return CBS_OK;
}

cbs_status cbs_export_mb_bsk(const cbs_context* ctx, uint64_t* out, size_t* words) {
    CBS_CHECK_ARG(ctx && words, "export_mb_bsk: null argument");
    if (ctx->br_mb <= 1 || !ctx->mb_ready) {
        set_error("export_mb_bsk: no grouped keys (select mb > 1 after cbs_keygen)");
        return CBS_ERR_NOT_READY;
    }
    *words = ctx->h_mbk.size();
    if (out) std::memcpy(out, ctx->h_mbk.data(), ctx->h_mbk.size() * sizeof(uint64_t));
    return CBS_OK;
}

cbs_status cbs_context_set_br_backend(cbs_context* ctx, int backend) {
    CBS_CHECK_ARG(ctx, "set_br_backend: null context");
    CBS_CHECK_ARG(backend == CBS_BR_NTT || backend == CBS_BR_FFT64 || backend == CBS_BR_FFT64_SPLIT,
                  "set_br_backend: unknown backend");
    if (backend == CBS_BR_FFT64 && (ctx->p.digits_g > 4 || ctx->p.base_g > (1u << 24))) {
        set_error("set_br_backend: the FFT64 backend supports at most 4 gadget digits of at most 24 bits");
        return CBS_ERR_UNSUPPORTED;
    }
    const int prev = ctx->br_backend;
    SplitPlan plan;
    if (backend == CBS_BR_FFT64_SPLIT) {
        // the grouping survives only a re-selection of the same backend
        if (cbs_status st = split_plan_for(ctx, prev == backend ? ctx->br_mb : 1, plan, "set_br_backend")) return st;
    }
    if (backend != prev && ctx->br_mb > 1) {  // grouped keys belong to the backend that made them
        ctx->br_mb = 1;
        ctx->mb_ready = false;
        ctx->h_mbk.clear();
        ctx->d_bskf_mb.reset();
        reset_split(ctx);
    }
    if (backend == CBS_BR_FFT64_SPLIT) {
        if (prev != backend || ctx->split.limbs != plan.limbs || ctx->split.limb_bits != plan.limb_bits)
            reset_split(ctx);
        ctx->split = plan;
        if (ctx->keys_ready) {
            if (cbs_status st = prepare_split(ctx)) return st;
        }
    } else if (ctx->split_ready) {  // the limb spectra are needed by the split backend only
        reset_split(ctx);
    }
    if (backend == CBS_BR_FFT64 && ctx->keys_ready) {
        if (cbs_status st = prepare_fft(ctx)) return st;
    }
    ctx->br_backend = backend;
    if (backend == CBS_BR_FFT64) {
        if (cbs_status st = apply_tuned_multibit(ctx)) return st;
    }
    if (backend != CBS_BR_NTT && ctx->br_method == CBS_BR_LMKCDEY) {  // LMKCDEY exists for the NTT form only
        ctx->br_method = CBS_BR_GINX;
        ctx->lmk_ready = false;
        ctx->h_lmk_eval.clear();
        ctx->h_lmk_auto.clear();
    }
    // captured AES round graphs bake in the kernel choice
    ctx->aes.drop_graphs();
    return CBS_OK;
}

cbs_status cbs_split_fft_plan(const cbs_params* params, uint32_t mb, uint32_t* limbs, uint32_t* limb_bits,
                              uint32_t* bound_bits) {
    CBS_CHECK_ARG(params && limbs && limb_bits && bound_bits, "split_fft_plan: null argument");
    CBS_CHECK_ARG(mb == 1 || mb == 2, "split_fft_plan: mb must be 1 or 2");
    if (cbs_status st = validate(*params)) return st;
    SplitPlan plan;
    if (!split_plan(params->N, params->Q, __builtin_ctz(params->base_g), params->digits_g, mb, plan)) {
        set_error("split_fft_plan: no split of at most 4 limbs keeps the products below 2^50 and Q/2");
        return CBS_ERR_UNSUPPORTED;
    }
    *limbs = plan.limbs;
    *limb_bits = plan.limb_bits;
    *bound_bits = plan.bound_bits;
    return CBS_OK;
}

cbs_status cbs_generate_mb_bsk_host(const cbs_params* params, uint64_t seed, uint32_t mb, uint64_t* out,
                                    size_t* words) {
    CBS_CHECK_ARG(params && words, "generate_mb_bsk_host: null argument");
    CBS_CHECK_ARG(mb >= 2 && mb <= 4, "generate_mb_bsk_host: mb must be 2, 3 or 4");
    if (cbs_status st = validate(*params)) return st;
    const size_t need = static_cast<size_t>((params->n + mb - 1) / mb) * mb_subsets(mb) * 2 * params->digits_g * 2 *
                        params->N;
    *words = need;
    if (!out) return CBS_OK;
    host::NttTables t;
    if (!host::make_ntt_tables(params->N, params->Q, t)) {
        set_error("generate_mb_bsk_host: NTT tables failed");
        return CBS_ERR_INVALID_ARG;
    }
    try {
        HostKeys k;
        generate_keys(*params, t, seed, k);
        std::vector<uint64_t> mbk;
        generate_mb_bsk(*params, t, k, mb, seed ^ kMbSeedTweak, mbk);
        std::memcpy(out, mbk.data(), mbk.size() * sizeof(uint64_t));
    } catch (const std::exception& e) {
        set_error(std::string("generate_mb_bsk_host: ") + e.what());
        return CBS_ERR_OOM;
    }
    return CBS_OK;
}

cbs_status cbs_generate_keys_host(const cbs_params* params, uint64_t seed, int32_t* s_lwe, int32_t* s_rlwe,
                                  uint64_t* bsk, uint64_t* ht, uint64_t* ss, uint16_t* ksk, uint64_t* tv,
                                  uint64_t* gpow, uint32_t* maps) {
    CBS_CHECK_ARG(params, "generate_keys_host: null params");
    if (cbs_status st = validate(*params)) return st;
    host::NttTables t;
    if (!host::make_ntt_tables(params->N, params->Q, t)) {
        set_error("generate_keys_host: NTT tables failed");
        return CBS_ERR_INVALID_ARG;
    }
    HostKeys k;
    try {
        generate_keys(*params, t, seed, k);
    } catch (const std::exception& e) {
        set_error(std::string("generate_keys_host: ") + e.what());
        return CBS_ERR_OOM;
    }
    auto cp = [](auto* dst, const auto& v) {
        if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(s_lwe, k.s_lwe);
    cp(s_rlwe, k.s_rlwe);
    cp(bsk, k.bsk);
    cp(ht, k.ht);
    cp(ss, k.ss);
    cp(ksk, k.ksk);
    cp(tv, k.tv);
    cp(gpow, k.gpow);
    cp(maps, k.maps);
    return CBS_OK;
}

cbs_status cbs_export_keys(const cbs_context* ctx, int32_t* s_lwe, int32_t* s_rlwe, uint64_t* bsk, uint64_t* ht,
                           uint64_t* ss, uint16_t* ksk, uint64_t* tv, uint64_t* gpow, uint32_t* maps) {
    CBS_CHECK_ARG(ctx, "export_keys: null context");
    if (!ctx->keys_ready) {
        set_error("export_keys: no keys (call cbs_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    const HostKeys& k = ctx->hk;
    auto cp = [](auto* dst, const auto& v) {
        if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(s_lwe, k.s_lwe);
    cp(s_rlwe, k.s_rlwe);
    cp(bsk, k.bsk);
    cp(ht, k.ht);
    cp(ss, k.ss);
    if (ksk && ctx->ksk_device_only) {
        // a device-generated key-switching key lives on the device only: unpad its rows
        const size_t row = (ctx->p.n + 1) * sizeof(uint16_t), stride = ksk_row_stride(ctx->p.n);
        CBS_CUDA_TRY(cudaSetDevice(ctx->device));
        CBS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        CBS_CUDA_TRY(cudaMemcpy2D(ksk, row, ctx->d_ksk.p, stride * sizeof(uint16_t), row, ctx->d_ksk.n / stride,
                                  cudaMemcpyDeviceToHost));
    } else {
        cp(ksk, k.ksk);
    }
    cp(tv, k.tv);
    cp(gpow, k.gpow);
    cp(maps, k.maps);
    return CBS_OK;
}

cbs_status cbs_context_tables(const cbs_context* ctx, const cbs_dmodulus** d_modulus, const uint64_t** d_twiddles,
                              const uint64_t** d_twiddles_shoup, const uint64_t** d_itwiddles,
                              const uint64_t** d_itwiddles_shoup, const uint64_t** d_n_inv,
                              const uint64_t** d_n_inv_shoup) {
    CBS_CHECK_ARG(ctx, "context_tables: null context");
    if (d_modulus) *d_modulus = ctx->d_mod.p;
    if (d_twiddles) *d_twiddles = ctx->d_rp.p;
    if (d_twiddles_shoup) *d_twiddles_shoup = ctx->d_rps.p;
    if (d_itwiddles) *d_itwiddles = ctx->d_irp.p;
    if (d_itwiddles_shoup) *d_itwiddles_shoup = ctx->d_irps.p;
    if (d_n_inv) *d_n_inv = ctx->d_ninv.p;
    if (d_n_inv_shoup) *d_n_inv_shoup = ctx->d_ninv_s.p;
    return CBS_OK;
}

static cbs_status need_keys(const cbs_context* c) {
    if (!c->keys_ready) {
        set_error("no key material (call cbs_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    return CBS_OK;
}

cbs_status cbs_blind_rotate_batch_device(cbs_context* ctx, const uint64_t* d_a, const uint64_t* d_b, uint32_t batch,
                                         uint32_t a_stride, uint64_t* d_mv, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "blind_rotate: null context");
    if (batch == 0) return CBS_OK;
    CBS_CHECK_ARG(d_a && d_b && d_mv, "blind_rotate: null pointer");
    CBS_CHECK_ARG(a_stride >= ctx->p.n, "blind_rotate: a_stride < n");
    if (cbs_status st = need_keys(ctx)) return st;
    return run_blind_rotate(ctx, d_a, d_b, batch, a_stride, d_mv, reinterpret_cast<cudaStream_t>(stream));
}

cbs_status cbs_trace_schemeswitch_device(cbs_context* ctx, const uint64_t* d_mv, uint32_t count, uint64_t* d_rgsw,
                                         cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "trace: null context");
    if (count == 0) return CBS_OK;
    CBS_CHECK_ARG(d_mv && d_rgsw, "trace: null pointer");
    if (cbs_status st = need_keys(ctx)) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (ctx->br_backend != CBS_BR_FFT64) return run_trace(ctx, d_mv, count, d_rgsw, s);
    // FFT backend: the MV RLWEs to the coefficient domain (context scratch), FFT HomTrace
    const size_t N = ctx->p.N, polys = static_cast<size_t>(count) * 2;
    CBS_CUDA_TRY(ctx->d_mv.alloc(polys * N));
    CBS_CUDA_TRY(ntt_inverse(ctx->d_mv.p, d_mv, nullptr, ctx->d_irp.p, ctx->d_irps.p, ctx->d_mod.p, ctx->d_ninv.p,
                             ctx->d_ninv_s.p, N, polys, s));
    return run_trace_fft_ntt_rows(ctx, ctx->d_mv.p, count, d_rgsw, s);
}

cbs_status cbs_circuit_bootstrap_batch_device(cbs_context* ctx, const uint64_t* d_a, const uint64_t* d_b,
                                              uint32_t batch, uint32_t a_stride, const uint64_t** d_rgsw_view,
                                              cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx && d_rgsw_view, "cbs: null argument");
    *d_rgsw_view = nullptr;
    if (batch == 0) return CBS_OK;
    CBS_CHECK_ARG(d_a && d_b, "cbs: null input");
    CBS_CHECK_ARG(a_stride >= ctx->p.n, "cbs: a_stride < n");
    if (batch > ctx->max_batch) {
        set_error("cbs: batch exceeds the context's max_batch (recreate the context)");
        return CBS_ERR_SHAPE_MISMATCH;
    }
    if (cbs_status st = need_keys(ctx)) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (cbs_status st = run_cbs(ctx, d_a, d_b, batch, a_stride, ctx->d_mv.p, ctx->d_rgsw.p, s)) return st;
    *d_rgsw_view = ctx->d_rgsw.p;
    return CBS_OK;
}

cbs_status cbs_circuit_bootstrap_batch(cbs_context* ctx, const uint64_t* h_a, const uint64_t* h_b, uint32_t batch,
                                       uint32_t a_stride, uint64_t* h_rgsw_out) {
    CBS_CHECK_ARG(ctx, "cbs_host: null context");
    if (batch == 0) return CBS_OK;
    CBS_CHECK_ARG(h_a && h_b && h_rgsw_out, "cbs_host: null pointer");
    CBS_CHECK_ARG(a_stride >= ctx->p.n, "cbs_host: a_stride < n");
    if (batch > ctx->max_batch) {
        set_error("cbs_host: batch exceeds the context's max_batch (recreate the context)");
        return CBS_ERR_SHAPE_MISMATCH;
    }
    const uint64_t q = ctx->p.q_lwe;
    for (size_t i = 0; i < static_cast<size_t>(batch); ++i) {
        CBS_CHECK_ARG(h_b[i] < q, "cbs_host: LWE b entries must be below q_lwe");
        for (uint32_t j = 0; j < ctx->p.n; ++j)
            CBS_CHECK_ARG(h_a[i * a_stride + j] < q, "cbs_host: LWE a entries must be below q_lwe");
    }
    if (cbs_status st = need_keys(ctx)) return st;
    cudaStream_t s = ctx->stream;
    DevBuf<uint64_t> d_a, d_b;
    CBS_CUDA_TRY(d_a.upload(h_a, static_cast<size_t>(batch) * a_stride, s));
    CBS_CUDA_TRY(d_b.upload(h_b, batch, s));
    if (cbs_status st = run_cbs(ctx, d_a.p, d_b.p, batch, a_stride, ctx->d_mv.p, ctx->d_rgsw.p, s)) return st;
    const size_t words = static_cast<size_t>(batch) * ctx->p.num_lut * 4 * ctx->p.N;
    CBS_CUDA_TRY(cudaMemcpyAsync(h_rgsw_out, ctx->d_rgsw.p, words * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    return CBS_OK;
}

cbs_status cbs_lut8x32_batch_device(cbs_context* ctx, const uint64_t* d_tables, uint32_t num_tables,
                                    const uint32_t* h_table_of_lut, const uint64_t* d_rgsw_all, uint32_t num_bits,
                                    uint64_t rgsw_stride, const uint32_t* h_ctrl_bits, uint32_t luts, uint64_t* d_out,
                                    cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "lut: null context");
    if (luts == 0) return CBS_OK;
    CBS_CHECK_ARG(d_tables && h_table_of_lut && d_rgsw_all && h_ctrl_bits && d_out, "lut: null pointer");
    CBS_CHECK_ARG(luts <= 65535, "lut: at most 65535 LUTs per call");
    CBS_CHECK_ARG(rgsw_stride >= static_cast<uint64_t>(ctx->p.num_lut) * 4 * ctx->p.N, "lut: rgsw_stride too small");
    for (uint32_t u = 0; u < luts; ++u) {
        CBS_CHECK_ARG(h_table_of_lut[u] < num_tables, "lut: table index out of range");
        for (uint32_t k = 0; k < 8; ++k)
            CBS_CHECK_ARG(h_ctrl_bits[u * 8 + k] < num_bits, "lut: control bit out of range");
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t N = ctx->p.N;
    CBS_CUDA_TRY(ctx->d_lut_sel_scratch.alloc(luts));
    CBS_CUDA_TRY(ctx->d_ctrl_scratch.alloc(static_cast<size_t>(luts) * 8));
    CBS_CUDA_TRY(ctx->d_lut_a.alloc(static_cast<size_t>(luts) * 128 * 2 * N));
    CBS_CUDA_TRY(ctx->d_lut_b.alloc(static_cast<size_t>(luts) * 64 * 2 * N));
    CBS_CUDA_TRY(cudaMemcpyAsync(ctx->d_lut_sel_scratch.p, h_table_of_lut, luts * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, s));
    CBS_CUDA_TRY(cudaMemcpyAsync(ctx->d_ctrl_scratch.p, h_ctrl_bits, static_cast<size_t>(luts) * 8 * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, s));
    return run_lut_levels(ctx, d_tables, 256ull * 2 * N, ctx->d_lut_sel_scratch.p, d_rgsw_all, rgsw_stride,
                          ctx->d_ctrl_scratch.p, luts, ctx->d_lut_a.p, ctx->d_lut_b.p, d_out, s);
}

cbs_status cbs_cmux_batch_device(cbs_context* ctx, const uint64_t* d_ct0, const uint64_t* d_ct1,
                                 const uint64_t* d_rgsw, uint64_t rgsw_stride, uint32_t count, uint64_t* d_out,
                                 cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "cmux: null context");
    if (count == 0) return CBS_OK;
    CBS_CHECK_ARG(d_ct0 && d_ct1 && d_rgsw && d_out, "cmux: null pointer");
    CBS_CHECK_ARG(count <= 65535, "cmux: at most 65535 CMuxes per call");
    const size_t N = ctx->p.N, L = ctx->p.num_lut, M = N / 2;
    CBS_CHECK_ARG(rgsw_stride == 0 || rgsw_stride >= L * 4 * N, "cmux: rgsw_stride below num_lut * 4 * N");
    const uint32_t n_rgsw = rgsw_stride == 0 ? 1u : count;  // stride 0: one control for every item
    if (ctx->br_backend == CBS_BR_FFT64 && !ctx->fft_ready) {
        set_error("cmux: FFT backend selected but its key material is not prepared");
        return CBS_ERR_NOT_READY;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // pairs [count][ct0, ct1][2][N] (the level-input layout of the LUT kernels), control u = bit u
    CBS_CUDA_TRY(ctx->d_lut_a.alloc(static_cast<size_t>(count) * 6 * N));
    uint64_t* pairs = ctx->d_lut_a.p;
    uint64_t* out_coef = pairs + static_cast<size_t>(count) * 4 * N;
    CBS_CUDA_TRY(cudaMemcpy2DAsync(pairs, 4 * N * 8, d_ct0, 2 * N * 8, 2 * N * 8, count, cudaMemcpyDeviceToDevice, s));
    CBS_CUDA_TRY(cudaMemcpy2DAsync(pairs + 2 * N, 4 * N * 8, d_ct1, 2 * N * 8, 2 * N * 8, count,
                                   cudaMemcpyDeviceToDevice, s));
    std::vector<uint32_t> ctrl(static_cast<size_t>(count) * 8, 0);
    for (uint32_t u = 0; u < count; ++u) ctrl[static_cast<size_t>(u) * 8] = u;
    CBS_CUDA_TRY(ctx->d_ctrl_scratch.upload(ctrl.data(), ctrl.size(), s));
    if (ctx->br_backend != CBS_BR_FFT64) {
        CmuxLevelArgs a{};
        a.t = ctx->ring();
        a.in_count = 2;
        a.in = pairs;
        a.in_lut_stride = 4 * N;
        a.lut_sel = nullptr;
        a.out = d_out;
        a.rgsw_all = d_rgsw;
        a.rgsw_stride = rgsw_stride;
        a.ctrl_bits = ctx->d_ctrl_scratch.p;
        a.level = 0;
        a.g = ctx->g_cc;
        a.digits = ctx->p.num_lut;
        CBS_CUDA_TRY(launch_cmux_level(a, ctx->p.N, count, s));
        return CBS_OK;
    }
    // FFT backend: inputs to the coefficient domain, control rows to spectra, the FFT CMux,
    // the output back to the NTT domain
    const size_t rows = static_cast<size_t>(n_rgsw) * L * 4;
    CBS_CUDA_TRY(ctx->d_lut_b.alloc(2 * rows * N));
    uint64_t* rgsw_coef = ctx->d_lut_b.p;
    double2* rgsw_spec = reinterpret_cast<double2*>(ctx->d_lut_b.p + rows * N);
    CBS_CUDA_TRY(ntt_inverse(pairs, pairs, nullptr, ctx->d_irp.p, ctx->d_irps.p, ctx->d_mod.p, ctx->d_ninv.p,
                             ctx->d_ninv_s.p, N, static_cast<size_t>(count) * 4, s));
    CBS_CUDA_TRY(cudaMemcpy2DAsync(rgsw_coef, L * 4 * N * 8, d_rgsw, (rgsw_stride ? rgsw_stride : L * 4 * N) * 8,
                                   L * 4 * N * 8, n_rgsw, cudaMemcpyDeviceToDevice, s));
    CBS_CUDA_TRY(ntt_inverse(rgsw_coef, rgsw_coef, nullptr, ctx->d_irp.p, ctx->d_irps.p, ctx->d_mod.p, ctx->d_ninv.p,
                             ctx->d_ninv_s.p, N, rows, s));
    const FftKeyArgs f = fft_key_args(ctx);
    CBS_CUDA_TRY(launch_coef_to_spectra(rgsw_coef, rgsw_spec, ctx->p.Q, f, ctx->p.N, rows, s));
    CmuxFftArgs a{};
    a.in = pairs;
    a.in_lut_stride = 4 * N;
    a.lut_sel = nullptr;
    a.out = out_coef;
    a.in_count = 2;
    a.rgswf = rgsw_spec;
    a.rgsw_stride = rgsw_stride ? L * 4 * M : 0;
    a.ctrl_bits = ctx->d_ctrl_scratch.p;
    a.level = 0;
    a.g = make_digit_prep(ctx->p.Q, ctx->g_cc, ctx->p.num_lut);
    a.digits = ctx->p.num_lut;
    a.in_spec = nullptr;
    CBS_CUDA_TRY(launch_cmux_level_fft(a, f, ctx->p.N, count, s));
    CBS_CUDA_TRY(ntt_forward(d_out, out_coef, ctx->d_rp.p, ctx->d_rps.p, ctx->d_mod.p, N,
                             static_cast<size_t>(count) * 2, s));
    return CBS_OK;
}

cbs_status cbs_extract_keyswitch_device(cbs_context* ctx, const uint64_t* d_words_coef, uint32_t words,
                                        const uint32_t* h_info, uint32_t count, uint64_t* d_out_a, uint64_t* d_out_b,
                                        uint32_t out_stride, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "extract: null context");
    if (count == 0) return CBS_OK;
    CBS_CHECK_ARG(d_words_coef && h_info && d_out_a && d_out_b, "extract: null pointer");
    CBS_CHECK_ARG(out_stride >= ctx->p.n, "extract: out_stride < n");
    CBS_CHECK_ARG(count <= 65535u, "extract: at most 65535 outputs per call");
    for (uint32_t t = 0; t < count; ++t) {
        CBS_CHECK_ARG((h_info[t] >> 16) < words && (h_info[t] & 0xFFFFu) < ctx->p.N, "extract: info out of range");
    }
    if (cbs_status st = need_keys(ctx)) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    CBS_CUDA_TRY(ctx->d_info_scratch.alloc(count));
    CBS_CUDA_TRY(cudaMemcpyAsync(ctx->d_info_scratch.p, h_info, count * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    return run_extract(ctx, d_words_coef, ctx->d_info_scratch.p, count, d_out_a, d_out_b, out_stride, s);
}

}  // extern "C"
