// gate_context.cuh -- the cbs_gate_context object behind the gate C ABI (gate.cu, gate_func.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/cbs_b200.h"
#include "common.cuh"
#include "devbuf.cuh"
#include "torus.cuh"

struct cbs_gate_context {
    cbs_gate_params p{};
    uint32_t max_batch = 0;
    bool keys_ready = false;
    std::vector<int32_t> s, z;      // LWE key (n), RLWE key (N), binary
    std::vector<uint32_t> bsk, ksk;  // coefficient form (exported) / device layout
    cbs::DevBuf<double2> d_bskf, d_tab;
    cbs::DevBuf<uint32_t> d_ksk, d_ext, d_tmp_a, d_tmp_b;
    // ragged plan (cbs_gate_ragged_plan): request table, its extracted-LWE scratch, grid
    cbs::DevBuf<cbs::GateReq> d_plan;
    cbs::DevBuf<uint32_t> d_plan_ext;
    uint32_t plan_reqs = 0, plan_items = 0, plan_grid = 0;
    // grouped (multi-bit) blind rotation: mb, its keys (coefficient form) and their spectra
    uint32_t br_mb = 1;
    bool mb_ready = false;
    uint64_t key_seed = 0;
    std::vector<uint32_t> mbk;
    cbs::DevBuf<double2> d_bskf_mb;
    // external-product arithmetic (CBS_FFT_*) and, for the FP32 modes, the key-limb spectra and
    // the FP32 transform table
    uint32_t fft_mode = CBS_FFT_FP64;
    bool f32_ready = false;
    cbs::DevBuf<float2> d_bskf32, d_tab32;
    // functional bootstrapping (gate_func.cu): the test vector [N], the torus form of the inputs
    // and the evaluator's intermediate ciphertexts [slots][max_batch][n + 1]
    cbs::DevBuf<uint32_t> d_tv, d_fin_a, d_fin_b, d_fwork;
};

namespace cbs {
// the key spectra / grouped keys / FP32 limbs of the context's current settings into a
cbs_status gate_fill_keys(const cbs_gate_context* ctx, GateArgs& a);
}  // namespace cbs
