// aes.cu -- homomorphic AES-128 CTR transciphering driver (device-resident rounds).
//
// Restates the reference's super-batch path (examples/aes_transcipher/main.cu:1318-1619):
// state bit t = byte*8 + b of each block starts as Enc(rk0 bit) + public counter bit * q/2
// (kernel_InitLWEStateFromRoundKey, gpu_lut.cuh:430); each round circuit-bootstraps all
// state bits into RGSW controls, evaluates the 16 T-table LUTs of every block as 256-leaf
// CMux trees (Te0..Te3, or Te4_* in round 10), assembles the four RLWE state words with
// the encrypted round-key word (column c gathers byte (row, c+row): ShiftRows), and
// extracts + key-switches the 128 state bits back to LWE (extract.cuh:283-366).  The
// per-round sequence of launches is captured once per chunk size into a CUDA graph.
#include <sys/random.h>

#include <cerrno>
#include <cstring>
#include <string>
#include <vector>

#include "aes_host.h"
#include "common.cuh"
#include "context.cuh"
#include "encrypt.cuh"

namespace cbs {

cudaError_t ntt_inverse(uint64_t* out, const uint64_t* in, const uint32_t* map, const uint64_t* itw,
                        const uint64_t* itws, const cbs_dmodulus* mod, const uint64_t* sc, const uint64_t* scs,
                        size_t dim, size_t batch, cudaStream_t s);

static constexpr uint32_t kAesMaxChunkBlocks = 256;

static cbs_status aes_prepare_chunk(cbs_context* c, uint32_t chunk) {
    AesState& A = c->aes;
    if (A.chunk_blocks >= chunk && A.ctr_bits.p) return CBS_OK;
    A.drop_graphs();
    const size_t N = c->p.N, n = c->p.n, L = c->p.num_lut;
    const size_t T = static_cast<size_t>(chunk) * 128, luts = static_cast<size_t>(chunk) * 16;
    CBS_CUDA_TRY(A.ctr_bits.alloc(T));
    CBS_CUDA_TRY(A.st_a.alloc(T * n));
    CBS_CUDA_TRY(A.st_b.alloc(T));
    CBS_CUDA_TRY(A.lut_a.alloc(luts * 128 * 2 * N));
    CBS_CUDA_TRY(A.lut_b.alloc(luts * 64 * 2 * N));
    CBS_CUDA_TRY(A.lut_out.alloc(luts * 2 * N));
    CBS_CUDA_TRY(A.words.alloc(static_cast<size_t>(chunk) * 4 * 2 * N));
    if (c->d_mv.n < T * L * 2 * N) CBS_CUDA_TRY(c->d_mv.alloc(T * L * 2 * N));
    if (c->d_rgsw.n < T * L * 4 * N) CBS_CUDA_TRY(c->d_rgsw.alloc(T * L * 4 * N));
    std::vector<uint32_t> sel0(luts), sel1(luts), ctrl(luts * 8), info(T);
    for (uint32_t blk = 0; blk < chunk; ++blk) {
        for (uint32_t row = 0; row < 4; ++row) {
            for (uint32_t col = 0; col < 4; ++col) {
                const uint32_t u = blk * 16 + row * 4 + col;
                sel0[u] = row;
                sel1[u] = 4 + row;
                const uint32_t byte = col * 4 + row;  // AesIndex(row, col)
                for (uint32_t k = 0; k < 8; ++k) ctrl[u * 8 + k] = blk * 128 + byte * 8 + k;
            }
        }
        for (uint32_t lt = 0; lt < 128; ++lt) {
            const uint32_t byte = lt / 8, b = lt % 8, col = byte / 4, row = byte % 4;
            const uint32_t bit_idx = (3 - row) * 8 + b;
            info[blk * 128 + lt] = ((blk * 4 + col) << 16) | bit_idx;
        }
    }
    cudaStream_t s = c->stream;
    CBS_CUDA_TRY(A.lut_sel[0].upload(sel0.data(), luts, s));
    CBS_CUDA_TRY(A.lut_sel[1].upload(sel1.data(), luts, s));
    CBS_CUDA_TRY(A.ctrl_bits.upload(ctrl.data(), ctrl.size(), s));
    CBS_CUDA_TRY(A.extract_info.upload(info.data(), info.size(), s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    A.chunk_blocks = chunk;
    return CBS_OK;
}

// one AES round on the resident chunk state (round in 1..10)
static cbs_status aes_round(cbs_context* c, uint32_t round, uint32_t chunk, cudaStream_t s) {
    AesState& A = c->aes;
    const uint32_t N = c->p.N, n = c->p.n, L = c->p.num_lut;
    const uint32_t T = chunk * 128, luts = chunk * 16;
    const bool final_round = (round == 10);
    if (c->br_backend == CBS_BR_FFT64) {
        // FFT path: MV RLWEs, LUT ciphertexts and words stay in the coefficient domain; the
        // RGSW controls are kept as row spectra in the RGSW buffer
        double2* rgswf = reinterpret_cast<double2*>(c->d_rgsw.p);
        if (cbs_status st = run_blind_rotate(c, A.st_a.p, A.st_b.p, T, n, c->d_mv.p, s, false)) return st;
        if (cbs_status st = run_trace_fft(c, c->d_mv.p, T * L, rgswf, s)) return st;
        if (cbs_status st = run_lut_levels_fft(c, A.tables_coef.p, 256ull * 2 * N, A.lut_sel[final_round ? 1 : 0].p,
                                               rgswf, static_cast<uint64_t>(L) * 4 * (N / 2), A.ctrl_bits.p, luts,
                                               A.lut_a.p, A.lut_b.p, A.lut_out.p, s, A.tables_spec.p))
            return st;
        CBS_CUDA_TRY(launch_assemble_words(A.words.p, A.lut_out.p,
                                           A.rk_words_coef.p + static_cast<size_t>(round) * 4 * 2 * N, c->p.Q, N,
                                           chunk, s));
        return run_extract(c, A.words.p, A.extract_info.p, T, A.st_a.p, A.st_b.p, n, s);
    }
    if (cbs_status st = run_blind_rotate(c, A.st_a.p, A.st_b.p, T, n, c->d_mv.p, s)) return st;
    if (cbs_status st = run_trace(c, c->d_mv.p, T * L, c->d_rgsw.p, s)) return st;
    if (cbs_status st = run_lut_levels(c, A.tables.p, 256ull * 2 * N, A.lut_sel[final_round ? 1 : 0].p, c->d_rgsw.p,
                                       static_cast<uint64_t>(L) * 4 * N, A.ctrl_bits.p, luts, A.lut_a.p, A.lut_b.p,
                                       A.lut_out.p, s))
        return st;
    CBS_CUDA_TRY(launch_assemble_words(A.words.p, A.lut_out.p, A.rk_words.p + static_cast<size_t>(round) * 4 * 2 * N,
                                       c->p.Q, N, chunk, s));
    CBS_CUDA_TRY(ntt_inverse(A.words.p, A.words.p, nullptr, c->d_irp.p, c->d_irps.p, c->d_mod.p, c->d_ninv.p,
                             c->d_ninv_s.p, N, static_cast<size_t>(chunk) * 8, s));
    return run_extract(c, A.words.p, A.extract_info.p, T, A.st_a.p, A.st_b.p, n, s);
}

static cbs_status aes_run_rounds(cbs_context* c, uint32_t chunk, cudaStream_t s, bool use_graphs) {
    AesState& A = c->aes;
    if (!use_graphs) {
        for (uint32_t r = 1; r <= 10; ++r)
            if (cbs_status st = aes_round(c, r, chunk, s)) return st;
        return CBS_OK;
    }
    if (A.graph_chunk != chunk) {
        A.drop_graphs();
        // this call runs eagerly (which also configures every kernel outside a capture);
        // the captured graphs serve the following calls
        for (uint32_t r = 1; r <= 10; ++r)
            if (cbs_status st = aes_round(c, r, chunk, s)) return st;
        for (uint32_t r = 1; r <= 10; ++r) {
            cudaGraph_t graph = nullptr;
            CBS_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            cbs_status st = aes_round(c, r, chunk, s);
            cudaError_t e = cudaStreamEndCapture(s, &graph);
            if (st != CBS_OK) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            CBS_CUDA_TRY(e);
            e = cudaGraphInstantiate(&A.graphs[r - 1], graph, 0);
            cudaGraphDestroy(graph);
            CBS_CUDA_TRY(e);
        }
        A.graph_chunk = chunk;
        return CBS_OK;
    }
    for (uint32_t r = 1; r <= 10; ++r) CBS_CUDA_TRY(cudaGraphLaunch(A.graphs[r - 1], s));
    return CBS_OK;
}

}  // namespace cbs

using namespace cbs;

extern "C" {

static cbs_status aes_derive_material(cbs_context* c);

// upload the host AES material of A (tables, round-key words, round-0 key bits) and derive
// the coefficient-domain copies of the FFT path
static cbs_status aes_upload_material(cbs_context* c) {
    AesState& A = c->aes;
    const uint32_t N = c->p.N;
    cudaStream_t s = c->stream;
    CBS_CUDA_TRY(A.tables.upload(A.h_tables.data(), A.h_tables.size(), s));
    CBS_CUDA_TRY(A.rk_words.upload(A.h_rk_words.data(), A.h_rk_words.size(), s));
    CBS_CUDA_TRY(A.rk0_a.upload(A.h_rk0_a.data(), A.h_rk0_a.size(), s));
    CBS_CUDA_TRY(A.rk0_b.upload(A.h_rk0_b.data(), A.h_rk0_b.size(), s));
    A.host_stale = false;
    return aes_derive_material(c);
}

// coefficient-domain copies of the device tables / round-key words (FFT path), then ready
static cbs_status aes_derive_material(cbs_context* c) {
    AesState& A = c->aes;
    const uint32_t N = c->p.N;
    cudaStream_t s = c->stream;
    const size_t tab_words = static_cast<size_t>(8) * 256 * 2 * N, rk_words = static_cast<size_t>(11) * 4 * 2 * N;
    CBS_CUDA_TRY(A.tables_coef.alloc(tab_words));
    CBS_CUDA_TRY(A.rk_words_coef.alloc(rk_words));
    CBS_CUDA_TRY(ntt_inverse(A.tables_coef.p, A.tables.p, nullptr, c->d_irp.p, c->d_irps.p, c->d_mod.p, c->d_ninv.p,
                             c->d_ninv_s.p, N, tab_words / N, s));
    CBS_CUDA_TRY(ntt_inverse(A.rk_words_coef.p, A.rk_words.p, nullptr, c->d_irp.p, c->d_irps.p, c->d_mod.p,
                             c->d_ninv.p, c->d_ninv_s.p, N, rk_words / N, s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    A.ready = true;
    A.spec_ready = false;
    return CBS_OK;
}

// level-0 table spectra of the FFT path (once per material; outside any capture)
static cbs_status aes_prepare_spectra(cbs_context* c, cudaStream_t s) {
    AesState& A = c->aes;
    if (c->br_backend != CBS_BR_FFT64 || A.spec_ready) return CBS_OK;
    const size_t M = c->p.N / 2, len = static_cast<size_t>(8) * 128 * 2 * c->p.num_lut * M;
    const double2* old = A.tables_spec.p;
    CBS_CUDA_TRY(A.tables_spec.alloc(len));
    if (A.tables_spec.p != old) A.drop_graphs();  // captured rounds hold the old pointer
    if (cbs_status st = build_table_spectra(c, A.tables_coef.p, 256ull * 2 * c->p.N, 8, A.tables_spec.p, s)) return st;
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    A.spec_ready = true;
    return CBS_OK;
}

cbs_status cbs_aes128_setup(cbs_context* ctx, const uint8_t* key, uint64_t seed) {
    CBS_CHECK_ARG(ctx && key, "aes_setup: null argument");
    if (!ctx->keys_ready) {
        set_error("aes_setup: no key material (call cbs_keygen first)");
        return CBS_ERR_NOT_READY;
    }
    if (!ctx->has_secret) {
        set_error("aes_setup: encrypting the AES material needs the secret key; the key owner's "
                  "cbs_aes128_export_material output loads with cbs_aes128_import_material");
        return CBS_ERR_NOT_READY;
    }
    cbs_context* c = ctx;
    AesState& A = c->aes;
    const uint32_t N = c->p.N, n = c->p.n;
    const uint64_t Q = c->p.Q, delta = Q >> 1;
    A.ready = false;  // set again once the new material is uploaded and derived
    aes::Block k{};
    std::memcpy(k.data(), key, 16);
    std::memcpy(A.key, key, 16);
    const auto rk = aes::key_expand(k);
    const auto te = aes::enc_tables();
    Rng rng(seed ^ 0x5eed5eed5eedull);
    std::vector<uint64_t> msg(N);
    // encrypted T-tables: word bits in coefficients 0..31, scaled by floor(Q/2)
    A.h_tables.assign(static_cast<size_t>(8) * 256 * 2 * N, 0);
    for (uint32_t tb = 0; tb < 8; ++tb)
        for (uint32_t x = 0; x < 256; ++x) {
            std::fill(msg.begin(), msg.end(), 0);
            for (uint32_t b = 0; b < 32; ++b) msg[b] = ((te[tb][x] >> b) & 1u) ? delta : 0;
            uint64_t* ct = A.h_tables.data() + (static_cast<size_t>(tb) * 256 + x) * 2 * N;
            rlwe_encrypt(c->p, c->tab, c->hk, rng, msg, ct, ct + N);
        }
    // encrypted round-key words (key_material.cuh:30-36)
    A.h_rk_words.assign(static_cast<size_t>(11) * 4 * 2 * N, 0);
    for (uint32_t r = 0; r <= 10; ++r)
        for (uint32_t col = 0; col < 4; ++col) {
            const uint32_t w =
                aes::pack_be(rk[r][col * 4 + 0], rk[r][col * 4 + 1], rk[r][col * 4 + 2], rk[r][col * 4 + 3]);
            std::fill(msg.begin(), msg.end(), 0);
            for (uint32_t b = 0; b < 32; ++b) msg[b] = ((w >> b) & 1u) ? delta : 0;
            uint64_t* ct = A.h_rk_words.data() + (static_cast<size_t>(r) * 4 + col) * 2 * N;
            rlwe_encrypt(c->p, c->tab, c->hk, rng, msg, ct, ct + N);
        }
    // encrypted round-0 key bits (LWE, q/2 scaling)
    A.h_rk0_a.assign(static_cast<size_t>(128) * n, 0);
    A.h_rk0_b.assign(128, 0);
    for (uint32_t t = 0; t < 128; ++t) {
        const uint32_t bit = (rk[0][t / 8] >> (t % 8)) & 1u;
        lwe_encrypt(c->p, c->hk, rng, bit ? (c->p.q_lwe >> 1) : 0, A.h_rk0_a.data() + static_cast<size_t>(t) * n,
                    A.h_rk0_b.data() + t);
    }
    return aes_upload_material(c);
}

// the plaintext words of the material: T-tables [8][256] then round-key words [11][4]
// (key_material.cuh:30-36), and the round-0 key bits [128]
static void aes_material_words(const uint8_t* key, std::vector<uint32_t>& words, std::vector<uint8_t>& bits) {
    aes::Block k{};
    std::memcpy(k.data(), key, 16);
    const auto rk = aes::key_expand(k);
    const auto te = aes::enc_tables();
    words.clear();
    for (uint32_t tb = 0; tb < 8; ++tb)
        for (uint32_t x = 0; x < 256; ++x) words.push_back(te[tb][x]);
    for (uint32_t r = 0; r <= 10; ++r)
        for (uint32_t col = 0; col < 4; ++col)
            words.push_back(aes::pack_be(rk[r][col * 4 + 0], rk[r][col * 4 + 1], rk[r][col * 4 + 2], rk[r][col * 4 + 3]));
    bits.resize(128);
    for (uint32_t t = 0; t < 128; ++t) bits[t] = (rk[0][t / 8] >> (t % 8)) & 1u;
}

// 32 bytes from the operating system's CSPRNG (getrandom(2), retried on EINTR / short reads)
static bool os_random_bytes(uint8_t* out, size_t len) {
    size_t got = 0;
    while (got < len) {
        const ssize_t r = getrandom(out + got, len - got, 0);
        if (r < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        got += static_cast<size_t>(r);
    }
    return true;
}

cbs_status cbs_aes128_setup_device(cbs_context* ctx, const uint8_t* key, const uint8_t* rng_key) {
    CBS_CHECK_ARG(ctx && key, "aes_setup_device: null argument");
    if (!ctx->keys_ready || !ctx->has_secret) {
        set_error("aes_setup_device: encrypting the AES material needs the secret key (cbs_keygen or "
                  "cbs_import_keys with secrets)");
        return CBS_ERR_NOT_READY;
    }
    cbs_context* c = ctx;
    AesState& A = c->aes;
    const uint32_t N = c->p.N, n = c->p.n;
    cudaStream_t s = c->stream;
    ChachaKey ck{};
    if (rng_key) {
        std::memcpy(ck.w, rng_key, 32);
    } else if (!os_random_bytes(reinterpret_cast<uint8_t*>(ck.w), 32)) {
        set_error(std::string("aes_setup_device: getrandom failed: ") + std::strerror(errno));
        return CBS_ERR_UNSUPPORTED;
    }
    // the buffers below are overwritten in place: until derive succeeds the context holds no
    // usable material (a failure midway leaves it not ready rather than half old, half new)
    A.ready = false;
    A.spec_ready = false;
    A.drop_graphs();
    std::memcpy(A.key, key, 16);
    std::vector<uint32_t> words;
    std::vector<uint8_t> bits;
    aes_material_words(key, words, bits);
    const uint32_t n_tab = 8 * 256, n_rk = 11 * 4;
    const auto cdt_r = cdt_table(c->p.sigma_rlwe), cdt_l = cdt_table(c->p.sigma_lwe);
    DevBuf<uint32_t> d_words;
    DevBuf<uint64_t> d_tmp, d_s_ntt, d_cdt_r, d_cdt_l;
    DevBuf<int32_t> d_s;
    DevBuf<uint8_t> d_bits;
    CBS_CUDA_TRY(d_words.upload(words.data(), words.size(), s));
    CBS_CUDA_TRY(d_s_ntt.upload(c->hk.s_ntt.data(), N, s));
    CBS_CUDA_TRY(d_s.upload(c->hk.s_lwe.data(), n, s));
    CBS_CUDA_TRY(d_bits.upload(bits.data(), 128, s));
    if (!cdt_r.empty()) CBS_CUDA_TRY(d_cdt_r.upload(cdt_r.data(), cdt_r.size(), s));
    if (!cdt_l.empty()) CBS_CUDA_TRY(d_cdt_l.upload(cdt_l.data(), cdt_l.size(), s));
    CBS_CUDA_TRY(d_tmp.alloc(static_cast<size_t>(n_tab) * N));
    CBS_CUDA_TRY(A.tables.alloc(static_cast<size_t>(n_tab) * 2 * N));
    CBS_CUDA_TRY(A.rk_words.alloc(static_cast<size_t>(n_rk) * 2 * N));
    CBS_CUDA_TRY(A.rk0_a.alloc(static_cast<size_t>(128) * n));
    CBS_CUDA_TRY(A.rk0_b.alloc(128));
    EncryptRlweArgs ra{};
    ra.key = ck;
    ra.tmp = d_tmp.p;
    ra.s_ntt = d_s_ntt.p;
    ra.cdt = d_cdt_r.p;
    ra.cdt_len = static_cast<uint32_t>(cdt_r.size());
    ra.N = N;
    ra.Q = c->p.Q;
    ra.delta = c->p.Q >> 1;
    ra.ratio0 = c->tab.ratio0;
    ra.ratio1 = c->tab.ratio1;
    ra.words = d_words.p;
    ra.ct = A.tables.p;
    ra.first = 0;
    CBS_CUDA_TRY(launch_encrypt_rlwe_words(ra, n_tab, c->d_rp.p, c->d_rps.p, c->d_mod.p, s));
    ra.words = d_words.p + n_tab;
    ra.ct = A.rk_words.p;
    ra.first = n_tab;
    CBS_CUDA_TRY(launch_encrypt_rlwe_words(ra, n_rk, c->d_rp.p, c->d_rps.p, c->d_mod.p, s));
    EncryptLweArgs la{};
    la.key = ck;
    la.bits = d_bits.p;
    la.s = d_s.p;
    la.cdt = d_cdt_l.p;
    la.cdt_len = static_cast<uint32_t>(cdt_l.size());
    la.n = n;
    la.a_stride = n;
    la.q = c->p.q_lwe;
    la.out_a = A.rk0_a.p;
    la.out_b = A.rk0_b.p;
    CBS_CUDA_TRY(launch_encrypt_lwe_bits(la, 128, s));
    // no host copies: cbs_aes128_export_material reads the device buffers
    A.h_tables.clear();
    A.h_rk_words.clear();
    A.h_rk0_a.clear();
    A.h_rk0_b.clear();
    A.host_stale = true;
    const cbs_status st = aes_derive_material(c);  // synchronizes before the scratch buffers are freed
    volatile uint32_t* wipe = ck.w;
    for (int i = 0; i < 8; ++i) wipe[i] = 0;
    return st;
}

cbs_status cbs_cdt_table_host(double sigma, uint64_t* out, uint32_t cap, uint32_t* len) {
    CBS_CHECK_ARG(len, "cdt_table: null len");
    CBS_CHECK_ARG(sigma >= 0 && sigma < 1e6, "cdt_table: sigma out of range");
    const auto T = cdt_table(sigma);
    *len = static_cast<uint32_t>(T.size());
    if (out) {
        CBS_CHECK_ARG(cap >= T.size(), "cdt_table: cap below the table length");
        std::memcpy(out, T.data(), T.size() * sizeof(uint64_t));
    }
    return CBS_OK;
}

cbs_status cbs_aes128_import_material(cbs_context* ctx, const uint64_t* h_tables, const uint64_t* h_rk_words,
                                      const uint64_t* h_rk0_a, const uint64_t* h_rk0_b) {
    CBS_CHECK_ARG(ctx && h_tables && h_rk_words && h_rk0_a && h_rk0_b, "aes_import: null argument");
    if (!ctx->keys_ready) {
        set_error("aes_import: import or generate the evaluation keys first");
        return CBS_ERR_NOT_READY;
    }
    cbs_context* c = ctx;
    AesState& A = c->aes;
    const uint32_t N = c->p.N, n = c->p.n;
    const uint64_t Q = c->p.Q, q = c->p.q_lwe;
    const size_t n_tab = static_cast<size_t>(8) * 256 * 2 * N, n_rk = static_cast<size_t>(11) * 4 * 2 * N;
    for (size_t i = 0; i < n_tab; ++i) CBS_CHECK_ARG(h_tables[i] < Q, "aes_import: table words must be below Q");
    for (size_t i = 0; i < n_rk; ++i) CBS_CHECK_ARG(h_rk_words[i] < Q, "aes_import: round-key words must be below Q");
    for (size_t i = 0; i < static_cast<size_t>(128) * n; ++i)
        CBS_CHECK_ARG(h_rk0_a[i] < q, "aes_import: round-0 LWE entries must be below q");
    for (size_t i = 0; i < 128; ++i) CBS_CHECK_ARG(h_rk0_b[i] < q, "aes_import: round-0 LWE entries must be below q");
    try {
        A.h_tables.assign(h_tables, h_tables + n_tab);
        A.h_rk_words.assign(h_rk_words, h_rk_words + n_rk);
        A.h_rk0_a.assign(h_rk0_a, h_rk0_a + static_cast<size_t>(128) * n);
        A.h_rk0_b.assign(h_rk0_b, h_rk0_b + 128);
    } catch (const std::exception& e) {
        set_error(std::string("aes_import: ") + e.what());
        return CBS_ERR_OOM;
    }
    std::memset(A.key, 0, sizeof(A.key));  // the AES key stays with its owner
    A.ready = false;
    return aes_upload_material(c);
}

cbs_status cbs_aes128_export_material(const cbs_context* ctx, uint64_t* h_tables, uint64_t* h_rk_words,
                                      uint64_t* h_rk0_a, uint64_t* h_rk0_b) {
    CBS_CHECK_ARG(ctx, "aes_export: null context");
    if (!ctx->aes.ready) {
        set_error("aes_export: call cbs_aes128_setup first");
        return CBS_ERR_NOT_READY;
    }
    const AesState& A = ctx->aes;
    if (A.host_stale) {  // encrypted on the device
        const size_t N = ctx->p.N, n = ctx->p.n;
        cudaStream_t s = ctx->stream;
        if (h_tables)
            CBS_CUDA_TRY(cudaMemcpyAsync(h_tables, A.tables.p, 8ull * 256 * 2 * N * 8, cudaMemcpyDeviceToHost, s));
        if (h_rk_words)
            CBS_CUDA_TRY(cudaMemcpyAsync(h_rk_words, A.rk_words.p, 11ull * 4 * 2 * N * 8, cudaMemcpyDeviceToHost, s));
        if (h_rk0_a) CBS_CUDA_TRY(cudaMemcpyAsync(h_rk0_a, A.rk0_a.p, 128ull * n * 8, cudaMemcpyDeviceToHost, s));
        if (h_rk0_b) CBS_CUDA_TRY(cudaMemcpyAsync(h_rk0_b, A.rk0_b.p, 128ull * 8, cudaMemcpyDeviceToHost, s));
        CBS_CUDA_TRY(cudaStreamSynchronize(s));
        return CBS_OK;
    }
    if (h_tables) std::memcpy(h_tables, A.h_tables.data(), A.h_tables.size() * 8);
    if (h_rk_words) std::memcpy(h_rk_words, A.h_rk_words.data(), A.h_rk_words.size() * 8);
    if (h_rk0_a) std::memcpy(h_rk0_a, A.h_rk0_a.data(), A.h_rk0_a.size() * 8);
    if (h_rk0_b) std::memcpy(h_rk0_b, A.h_rk0_b.data(), A.h_rk0_b.size() * 8);
    return CBS_OK;
}

cbs_status cbs_aes128_ctr_transcipher_device(cbs_context* ctx, const uint8_t* d_counter_bits, uint32_t blocks,
                                             uint64_t* d_out_a, uint64_t* d_out_b, int use_graphs,
                                             cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "aes_transcipher: null context");
    if (blocks == 0) return CBS_OK;
    CBS_CHECK_ARG(d_counter_bits && d_out_a && d_out_b, "aes_transcipher: null pointer");
    if (!ctx->aes.ready) {
        set_error("aes_transcipher: call cbs_aes128_setup first");
        return CBS_ERR_NOT_READY;
    }
    cbs_context* c = ctx;
    AesState& A = c->aes;
    cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : c->stream;
    const uint32_t n = c->p.n;
    const uint32_t max_chunk = std::max(1u, std::min(kAesMaxChunkBlocks, c->max_batch / 128u));
    const uint32_t chunk = std::min(blocks, max_chunk);
    if (cbs_status st = aes_prepare_chunk(c, chunk)) return st;
    if (cbs_status st = aes_prepare_spectra(c, s)) return st;
    for (uint32_t off = 0; off < blocks; off += chunk) {
        const uint32_t cur = std::min(chunk, blocks - off);
        const uint32_t T = cur * 128;
        CBS_CUDA_TRY(launch_init_state(A.st_a.p, A.st_b.p, A.rk0_a.p, A.rk0_b.p,
                                       d_counter_bits + static_cast<size_t>(off) * 128,
                                       c->p.q_lwe >> 1, c->p.q_lwe, n, T, s));
        // graphs are built for full chunks; a ragged tail runs eagerly
        if (cbs_status st = aes_run_rounds(c, cur, s, use_graphs && cur == chunk)) return st;
        CBS_CUDA_TRY(cudaMemcpyAsync(d_out_a + static_cast<size_t>(off) * 128 * n, A.st_a.p,
                                     static_cast<size_t>(T) * n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        CBS_CUDA_TRY(cudaMemcpyAsync(d_out_b + static_cast<size_t>(off) * 128, A.st_b.p,
                                     static_cast<size_t>(T) * sizeof(uint64_t),
                                     cudaMemcpyDeviceToDevice, s));
    }
    return CBS_OK;
}

cbs_status cbs_aes128_ctr_add_ciphertext_device(cbs_context* ctx, const uint8_t* d_cipher, uint32_t blocks,
                                               uint64_t* d_b, cbs_stream_t stream) {
    CBS_CHECK_ARG(ctx, "aes_add_ciphertext: null context");
    if (blocks == 0) return CBS_OK;
    CBS_CHECK_ARG(d_cipher && d_b, "aes_add_ciphertext: null pointer");
    CBS_CHECK_ARG(blocks <= (1u << 24), "aes_add_ciphertext: at most 2^24 blocks per call");
    cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->stream;
    CBS_CUDA_TRY(launch_add_public_bits(d_b, d_cipher, ctx->p.q_lwe >> 1, ctx->p.q_lwe, blocks * 128u, s));
    return CBS_OK;
}

// host transciphering: keystream LWEs of AES_K(counter), plus the public ciphertext bits
// when h_cipher is given (then LWEs of the plaintext bits)
static cbs_status aes_ctr_host(cbs_context* ctx, const uint8_t* h_counters, const uint8_t* h_cipher,
                               uint32_t blocks, uint64_t* h_out_a, uint64_t* h_out_b) {
    cbs_context* c = ctx;
    cudaStream_t s = c->stream;
    const size_t T = static_cast<size_t>(blocks) * 128, n = c->p.n;
    std::vector<uint8_t> bits(T);
    for (size_t blk = 0; blk < blocks; ++blk)
        for (uint32_t t = 0; t < 128; ++t) bits[blk * 128 + t] = (h_counters[blk * 16 + t / 8] >> (t % 8)) & 1u;
    // staging buffers kept by the context across calls (grown on demand)
    AesState& A = c->aes;
    DevBuf<uint8_t>& d_bits = A.host_bits;
    DevBuf<uint64_t>&d_a = A.host_a, &d_b = A.host_b;
    CBS_CUDA_TRY(d_bits.upload(bits.data(), T, s));
    CBS_CUDA_TRY(d_a.alloc(T * n));
    CBS_CUDA_TRY(d_b.alloc(T));
    if (cbs_status st = cbs_aes128_ctr_transcipher_device(c, d_bits.p, blocks, d_a.p, d_b.p, 1,
                                                          reinterpret_cast<cbs_stream_t>(s)))
        return st;
    DevBuf<uint8_t>& d_cipher = A.host_cipher;
    if (h_cipher) {
        CBS_CUDA_TRY(d_cipher.upload(h_cipher, static_cast<size_t>(blocks) * 16, s));
        if (cbs_status st = cbs_aes128_ctr_add_ciphertext_device(c, d_cipher.p, blocks, d_b.p,
                                                                 reinterpret_cast<cbs_stream_t>(s)))
            return st;
    }
    CBS_CUDA_TRY(cudaMemcpyAsync(h_out_a, d_a.p, T * n * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CBS_CUDA_TRY(cudaMemcpyAsync(h_out_b, d_b.p, T * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    return CBS_OK;
}

cbs_status cbs_aes128_ctr_transcipher(cbs_context* ctx, const uint8_t* h_counters, uint32_t blocks, uint64_t* h_out_a,
                                      uint64_t* h_out_b) {
    CBS_CHECK_ARG(ctx, "aes_transcipher: null context");
    if (blocks == 0) return CBS_OK;
    CBS_CHECK_ARG(h_counters && h_out_a && h_out_b, "aes_transcipher: null pointer");
    return aes_ctr_host(ctx, h_counters, nullptr, blocks, h_out_a, h_out_b);
}

cbs_status cbs_aes128_ctr_transcipher_ciphertext(cbs_context* ctx, const uint8_t* h_counters,
                                                 const uint8_t* h_cipher, uint32_t blocks, uint64_t* h_out_a,
                                                 uint64_t* h_out_b) {
    CBS_CHECK_ARG(ctx, "aes_transcipher: null context");
    if (blocks == 0) return CBS_OK;
    CBS_CHECK_ARG(h_counters && h_cipher && h_out_a && h_out_b, "aes_transcipher: null pointer");
    return aes_ctr_host(ctx, h_counters, h_cipher, blocks, h_out_a, h_out_b);
}

cbs_status cbs_lwe_decrypt_bits(const cbs_context* ctx, const uint64_t* h_a, const uint64_t* h_b, uint32_t count,
                                uint32_t a_stride, uint8_t* h_bits) {
    CBS_CHECK_ARG(ctx && (count == 0 || (h_a && h_b && h_bits)), "lwe_decrypt: null argument");
    if (!ctx->keys_ready || !ctx->has_secret) {
        set_error("lwe_decrypt: no secret key in this context");
        return CBS_ERR_NOT_READY;
    }
    CBS_CHECK_ARG(a_stride >= ctx->p.n, "lwe_decrypt: a_stride < n");
    const uint64_t q = ctx->p.q_lwe;
    for (uint32_t t = 0; t < count; ++t) {
        unsigned __int128 dot = 0;
        for (uint32_t i = 0; i < ctx->p.n; ++i)
            if (ctx->hk.s_lwe[i]) dot += h_a[static_cast<size_t>(t) * a_stride + i];
        const uint64_t ph = static_cast<uint64_t>((static_cast<unsigned __int128>(h_b[t]) + q - dot % q) % q);
        // round(2 * phase / q) mod 2
        h_bits[t] = static_cast<uint8_t>(((2 * ph + q / 2) / q) & 1u);
    }
    return CBS_OK;
}

}  // extern "C"
