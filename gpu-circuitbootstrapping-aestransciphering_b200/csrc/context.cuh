// context.cuh -- the cbs_context object behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <memory>
#include <vector>

#include "../../include/cbs_b200.h"
#include "cbs_kernels.cuh"
#include "devbuf.cuh"
#include "encrypt.cuh"
#include "extract_kernels.cuh"
#include "fft_kernels.cuh"
#include "host_math.h"
#include "keygen.h"

namespace cbs {

struct AesState {
    bool ready = false;
    bool host_stale = false;              // material encrypted on the device: no h_* copies
    uint8_t key[16];
    uint32_t chunk_blocks = 0;            // blocks per device chunk
    DevBuf<uint64_t> tables;              // [8][256][2][N]  Te0..3, Te4_0..3
    DevBuf<uint64_t> rk_words;            // [11][4][2][N]
    // coefficient-domain copies of tables and rk_words for the FFT CMux path, and the level-0
    // digit spectra of the table pairs ([8][128][2*num_lut][N/2], built on first FFT use)
    DevBuf<uint64_t> tables_coef, rk_words_coef;
    DevBuf<double2> tables_spec;
    bool spec_ready = false;
    DevBuf<uint64_t> rk0_a, rk0_b;        // [128][n], [128]
    std::vector<uint64_t> h_tables, h_rk_words, h_rk0_a, h_rk0_b;
    // per-chunk workspace
    DevBuf<uint8_t> ctr_bits;             // [chunk*128]
    DevBuf<uint64_t> st_a, st_b;          // [chunk*128][n], [chunk*128]
    DevBuf<uint64_t> lut_a, lut_b;        // ping-pong level buffers
    DevBuf<uint64_t> lut_out;             // [chunk*16][2][N]
    DevBuf<uint64_t> words;               // [chunk*4][2][N]
    DevBuf<uint32_t> lut_sel[2];          // table id per LUT (normal rounds, final round)
    DevBuf<uint32_t> ctrl_bits;           // [chunk*16][8]
    DevBuf<uint32_t> extract_info;        // [chunk*128]
    // staging of the host-buffer entry points (counter bits, outputs, public ciphertext)
    DevBuf<uint8_t> host_bits, host_cipher;
    DevBuf<uint64_t> host_a, host_b;
    std::array<cudaGraphExec_t, 10> graphs{};
    uint32_t graph_chunk = 0;
    // the captured round graphs hold device pointers of the keys; dropped when keys change
    void drop_graphs() {
        for (auto& g : graphs)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        graph_chunk = 0;
    }
};

}  // namespace cbs

struct cbs_context {
    cbs_params p{};
    uint32_t max_batch = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    cbs::host::NttTables tab;
    cbs::Gadget g_br{}, g_cc{}, g_ht{}, g_ss{};
    uint32_t rounds = 0, bitwidth = 0;
    uint64_t qneg_inv = 0, one_s = 0, mont_r = 0;
    // device tables
    cbs::DevBuf<uint64_t> d_rp, d_rps, d_irp, d_irps, d_ninv, d_ninv_s;
    cbs::DevBuf<cbs_dmodulus> d_mod;
    cbs::DevBuf<uint32_t> d_maps;
    // keys (has_secret: hk holds s_lwe / s_rlwe, i.e. the keys came from cbs_keygen or were
    // imported with their secrets; without them the context evaluates only)
    bool keys_ready = false;
    bool has_secret = false;
    cbs::HostKeys hk;
    cbs::DevBuf<uint64_t> d_tv, d_gadd, d_bsk, d_ht, d_ss;
    cbs::DevBuf<uint16_t> d_ksk;
    // FP64 FFT blind-rotation backend (built on demand from the keys)
    int br_backend = 0;  // CBS_BR_NTT, CBS_BR_FFT64 or CBS_BR_FFT64_SPLIT
    bool fft_ready = false;
    cbs::DevBuf<double2> d_bskf, d_fft_tab;
    cbs::DevBuf<double2> d_htf, d_ssf;  // HomTrace / SchemeSwitch key spectra
    // exact split-FFT blind rotation (CBS_BR_FFT64_SPLIT): key limb spectra and the limb plan
    bool split_ready = false;
    cbs::SplitPlan split{};
    cbs::DevBuf<double2> d_bskx;
    // multi-bit blind rotation (FFT backend): 1 = one coefficient per step, 2 or 3 = grouped
    uint32_t br_mb = 1;
    bool mb_explicit = false;            // mb chosen by the caller (not by the tuning cache)
    uint32_t br_schedule = 0;            // CBS_BR_SCHEDULE_*
    bool has_tuned = false;              // a tuning-cache entry for this GPU and parameter set
    cbs_tune_choice tuned{};
    bool mb_ready = false;
    uint64_t key_seed = 0;
    bool device_keyed = false;           // keys drawn on the device (cbs_keygen_device) under keygen_key
    bool ksk_device_only = false;        // the key-switching key exists only in d_ksk (hk.ksk empty)
    cbs::ChachaKey keygen_key{};
    std::vector<uint64_t> h_mbk;         // grouped keys, NTT domain (kept for export)
    cbs::DevBuf<double2> d_bskf_mb;      // their spectra
    // LMKCDEY blind rotation (NTT backend): the keys in the NTT domain (kept for export), their
    // Montgomery-form device copies, the automorphism maps and the discrete-log table
    int br_method = 0;                   // CBS_BR_GINX or CBS_BR_LMKCDEY
    uint32_t lmk_num_auto = 0;
    uint32_t lmk_window = 0;             // > 1: the windowed key set (5^1 .. 5^w, 5^2w, 5^3w, ...)
    bool lmk_ready = false;
    std::vector<uint64_t> h_lmk_eval, h_lmk_auto;
    cbs::DevBuf<uint64_t> d_lmk_eval, d_lmk_auto;
    cbs::DevBuf<uint32_t> d_lmk_maps;
    cbs::DevBuf<int32_t> d_lmk_log;
    cbs::DevBuf<uint64_t> d_pow2, d_pow2s;
    // scratch
    cbs::DevBuf<uint64_t> d_mv, d_rgsw;
    cbs::DevBuf<uint32_t> d_info_scratch, d_lut_sel_scratch, d_ctrl_scratch;
    cbs::DevBuf<uint64_t> d_lut_a, d_lut_b;
    cbs::AesState aes;

    cbs::RingTables ring() const {
        cbs::RingTables t;
        t.rp = d_rp.p;
        t.rps = d_rps.p;
        t.irp = d_irp.p;
        t.irps = d_irps.p;
        t.q = p.Q;
        t.n_inv = tab.n_inv;
        t.n_inv_s = tab.n_inv_sh;
        t.ratio0 = tab.ratio0;
        t.ratio1 = tab.ratio1;
        t.qneg_inv = qneg_inv;
        t.one_s = one_s;
        return t;
    }
};

namespace cbs {
// shared entry used by the AES driver and the C ABI
// mv_ntt = false (FFT backend only) leaves the MV RLWEs in the coefficient domain
cbs_status run_blind_rotate(cbs_context* c, const uint64_t* d_a, const uint64_t* d_b, uint32_t batch,
                            uint32_t a_stride, uint64_t* d_mv, cudaStream_t s, bool mv_ntt = true);
FftKeyArgs fft_key_args(const cbs_context* c);
// the tuning cache (tune.cu): the entry for this context's GPU and parameter set, if any
bool tune_cache_lookup(const cbs_context* c, const char* path, cbs_tune_choice* out);
// on the FFT64 backend, switch to the tuning cache's grouping unless the caller chose one (grouped
// keys are generated from the secret key; without it the grouping stays as it is)
cbs_status apply_tuned_multibit(cbs_context* c);
// host key copies (c->hk) -> device keys, derived tables; resets the FFT / grouped state
cbs_status upload_host_keys(cbs_context* c);
// the derived tables (tv, gadd, maps) of c->hk to the device and the key state reset, after the
// key material itself is on the device (upload_host_keys or the device keygen)
cbs_status finish_key_upload(cbs_context* c);
// the grouped keys of a device-generated key set into c->h_mbk (keygen_device.cu)
cbs_status device_grouped_keys(cbs_context* c, uint32_t mb);
// parameter checks of cbs_context_create
cbs_status validate_params(const cbs_params& p);
// LMKCDEY (lmkcdey.cu): its keys from the context's secrets when the method is selected and keys
// exist; the blind rotation into the MV layout of run_blind_rotate (NTT domain)
cbs_status prepare_lmkcdey(cbs_context* c);
cbs_status run_blind_rotate_lmkcdey(cbs_context* c, const uint64_t* d_a, const uint64_t* d_b, uint32_t batch,
                                    uint32_t a_stride, uint64_t* d_mv, cudaStream_t s);
// blind rotation + HomTrace/SchemeSwitch of the selected backend: LWE -> RGSW rows in the
// NTT-domain reference layout [batch][num_lut][2][2][N]; d_mv is [batch][num_lut][2][N] scratch
// FFT HomTrace + SchemeSwitch with the rows converted to the NTT-domain reference layout
cbs_status run_trace_fft_ntt_rows(cbs_context* c, const uint64_t* d_mv_coef, uint32_t count, uint64_t* d_rgsw,
                                  cudaStream_t s);
cbs_status run_cbs(cbs_context* c, const uint64_t* d_a, const uint64_t* d_b, uint32_t batch, uint32_t a_stride,
                   uint64_t* d_mv, uint64_t* d_rgsw, cudaStream_t s);
// FFT HomTrace + SchemeSwitch: coefficient-domain MV RLWEs -> RGSW row spectra [count][2][2][N/2]
cbs_status run_trace_fft(cbs_context* c, const uint64_t* d_mv_coef, uint32_t count, double2* d_rgswf,
                         cudaStream_t s);
// the 8 FFT CMux levels of the LUT trees, coefficient-domain tables in and outputs out
// d_table_spec (optional): the level-0 pair spectra of d_tables (build_table_spectra)
cbs_status run_lut_levels_fft(cbs_context* c, const uint64_t* d_tables, uint64_t table_stride,
                              const uint32_t* d_lut_sel, const double2* d_rgswf, uint64_t rgsw_stride,
                              const uint32_t* d_ctrl, uint32_t luts, uint64_t* d_buf_a, uint64_t* d_buf_b,
                              uint64_t* d_out, cudaStream_t s, const double2* d_table_spec = nullptr);
// level-0 digit spectra of `sets` fixed 256-entry tables (coefficient domain) into out
// [sets][128][2*num_lut][N/2]
cbs_status build_table_spectra(cbs_context* c, const uint64_t* d_tables, uint64_t table_stride, uint32_t sets,
                               double2* out, cudaStream_t s);
cbs_status run_trace(cbs_context* c, const uint64_t* d_mv, uint32_t count, uint64_t* d_rgsw, cudaStream_t s);
cbs_status run_lut_levels(cbs_context* c, const uint64_t* d_tables, uint64_t table_stride, const uint32_t* d_lut_sel,
                          const uint64_t* d_rgsw_all, uint64_t rgsw_stride, const uint32_t* d_ctrl, uint32_t luts,
                          uint64_t* d_buf_a, uint64_t* d_buf_b, uint64_t* d_out, cudaStream_t s);
cbs_status run_extract(cbs_context* c, const uint64_t* d_words_coef, const uint32_t* d_info, uint32_t count,
                       uint64_t* d_out_a, uint64_t* d_out_b, uint32_t out_stride, cudaStream_t s);
}  // namespace cbs
