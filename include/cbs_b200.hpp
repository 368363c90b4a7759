// cbs_b200.hpp -- header-only C++ facade with the reference's call shapes.
//
// Mirrors the interfaces a caller of the reference binds for this path:
//   * Phantom's 1-D NTT functions (include/ntt.cuh:215-227): same names and argument order,
//     DModulus -> cbs_dmodulus (identical layout), cudaStream_t by const reference;
//   * GPUCirBTSContext (bitwise/include/cirbts/cirbts.cuh:420-498): construction from
//     parameters + max batch, the device-LWE circuit-bootstrapping entry point returning a
//     non-owning DeviceRGSWBatchView, the NTT-table accessors and stream();
//   * the example's LUT and extraction helpers (gpu_lut.cuh:1783, extract.cuh:283).
// Errors surface as exceptions on this side (like OPENFHE_THROW / PHANTOM_CHECK_CUDA in the
// reference); the C ABI underneath never throws.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "cbs_b200.h"

namespace cbs_b200 {

class Error : public std::runtime_error {
   public:
    Error(cbs_status s, const std::string& where)
        : std::runtime_error(where + ": status " + std::to_string(static_cast<int>(s)) + ": " + cbs_last_error()),
          status(s) {}
    cbs_status status;
};

inline void check(cbs_status s, const char* where) {
    if (s != CBS_OK) throw Error(s, where);
}

inline cbs_stream_t as_stream(const cudaStream_t& s) { return reinterpret_cast<cbs_stream_t>(s); }

// ---- Phantom 1-D NTT (include/ntt.cuh:215-227) ----
inline void fnwt_1d_opt_batched(uint64_t* inout, const uint64_t* twiddles, const uint64_t* twiddles_shoup,
                                const cbs_dmodulus* modulus, size_t dim, size_t batch, const cudaStream_t& stream) {
    check(cbs_fnwt_1d_opt_batched(inout, twiddles, twiddles_shoup, modulus, dim, batch, as_stream(stream)),
          "fnwt_1d_opt_batched");
}

inline void inwt_1d_opt_batched(uint64_t* inout, const uint64_t* itwiddles, const uint64_t* itwiddles_shoup,
                                const cbs_dmodulus* modulus, const uint64_t* scalar, const uint64_t* scalar_shoup,
                                size_t dim, size_t batch, const cudaStream_t& stream) {
    check(cbs_inwt_1d_opt_batched(inout, itwiddles, itwiddles_shoup, modulus, scalar, scalar_shoup, dim, batch,
                                  as_stream(stream)),
          "inwt_1d_opt_batched");
}

inline void inwt_1d_opt_outofplace_batched(uint64_t* out, const uint64_t* in, const uint64_t* itwiddles,
                                           const uint64_t* itwiddles_shoup, const cbs_dmodulus* modulus,
                                           const uint64_t* scalar, const uint64_t* scalar_shoup, size_t dim,
                                           size_t batch, const cudaStream_t& stream) {
    check(cbs_inwt_1d_opt_outofplace_batched(out, in, itwiddles, itwiddles_shoup, modulus, scalar, scalar_shoup, dim,
                                             batch, as_stream(stream)),
          "inwt_1d_opt_outofplace_batched");
}

inline void inwt_1d_opt_permute_batched(uint64_t* out, const uint64_t* in, const uint32_t* map,
                                        const uint64_t* itwiddles, const uint64_t* itwiddles_shoup,
                                        const cbs_dmodulus* modulus, const uint64_t* scalar,
                                        const uint64_t* scalar_shoup, size_t dim, size_t batch,
                                        const cudaStream_t& stream) {
    check(cbs_inwt_1d_opt_permute_batched(out, in, map, itwiddles, itwiddles_shoup, modulus, scalar, scalar_shoup, dim,
                                          batch, as_stream(stream)),
          "inwt_1d_opt_permute_batched");
}

// ---- GPUCirBTSContext (bitwise/include/cirbts/cirbts.cuh:31-500) ----
class GPUCirBTSContext {
   public:
    // Non-owning view (cirbts.cuh:406-418): per ciphertext [digitsCC*2 rows][2 polys][N].
    struct DeviceRGSWBatchView {
        const uint64_t* d_rgsw{};
        uint32_t batch{};
        uint32_t digitsCC{};
        uint32_t N{};
        size_t per_ciphertext_elems{};
        cudaStream_t stream{};
    };

    explicit GPUCirBTSContext(const cbs_params& params, uint32_t maxBatchSize = 1)
        : params_(params), max_batch_(maxBatchSize ? maxBatchSize : 1) {
        check(cbs_context_create(&params_, max_batch_, &ctx_), "GPUCirBTSContext");
    }
    GPUCirBTSContext(const GPUCirBTSContext&) = delete;
    GPUCirBTSContext& operator=(const GPUCirBTSContext&) = delete;
    ~GPUCirBTSContext() { cbs_context_destroy(ctx_); }

    // KeyGen + RLWEKeyGen + CirBTKeyGen + KeySwitchGen of the example, from a seed
    void KeyGen(uint64_t seed) { check(cbs_keygen(ctx_, seed), "KeyGen"); }

    [[nodiscard]] const cbs_dmodulus* d_modulus() const { return table(0); }
    [[nodiscard]] const uint64_t* d_twiddles() const { return tab64(1); }
    [[nodiscard]] const uint64_t* d_twiddles_shoup() const { return tab64(2); }
    [[nodiscard]] const uint64_t* d_itwiddles() const { return tab64(3); }
    [[nodiscard]] const uint64_t* d_itwiddles_shoup() const { return tab64(4); }
    [[nodiscard]] const uint64_t* d_n_inv_mod_q() const { return tab64(5); }
    [[nodiscard]] const uint64_t* d_n_inv_mod_q_shoup() const { return tab64(6); }
    [[nodiscard]] cudaStream_t stream() const {
        cbs_stream_t s{};
        check(cbs_context_stream(ctx_, &s), "stream");
        return reinterpret_cast<cudaStream_t>(s);
    }

    // cirbts-batch.cu:1416 gpu_CircuitBootstrappingBatchToDeviceFromDeviceLWE
    [[nodiscard]] DeviceRGSWBatchView gpu_CircuitBootstrappingBatchToDeviceFromDeviceLWE(const uint64_t* d_a,
                                                                                       const uint64_t* d_b,
                                                                                       uint32_t batch,
                                                                                       uint32_t a_stride) const {
        DeviceRGSWBatchView v{};
        if (!d_a || !d_b || batch == 0) return v;
        const uint64_t* p = nullptr;
        const cudaStream_t s = stream();
        check(cbs_circuit_bootstrap_batch_device(ctx_, d_a, d_b, batch, a_stride, &p, as_stream(s)),
              "gpu_CircuitBootstrappingBatchToDeviceFromDeviceLWE");
        v.d_rgsw = p;
        v.batch = batch;
        v.digitsCC = params_.num_lut;
        v.N = params_.N;
        v.per_ciphertext_elems = static_cast<size_t>(params_.num_lut) * 4 * params_.N;
        v.stream = s;
        return v;
    }

    [[nodiscard]] cbs_context* handle() const { return ctx_; }
    [[nodiscard]] const cbs_params& params() const { return params_; }

   private:
    const cbs_dmodulus* table(int) const {
        const cbs_dmodulus* m = nullptr;
        check(cbs_context_tables(ctx_, &m, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr), "tables");
        return m;
    }
    const uint64_t* tab64(int which) const {
        const uint64_t* t[6] = {};
        check(cbs_context_tables(ctx_, nullptr, &t[0], &t[1], &t[2], &t[3], &t[4], &t[5]), "tables");
        return t[which - 1];
    }
    cbs_params params_;
    uint32_t max_batch_;
    cbs_context* ctx_ = nullptr;
};

// ---- Phantom RNS core (include/context.cuh:161, include/ntt.cuh:232-262,
//      src/eval_key_switch.cu:94) ----
// Owns the modulus chain Q || P and its device tables (PhantomContext's gpu_rns_tables()).
class RnsContext {
   public:
    RnsContext(uint32_t poly_degree, const std::vector<uint64_t>& q, const std::vector<uint64_t>& p)
        : size_q_(static_cast<uint32_t>(q.size())), size_p_(static_cast<uint32_t>(p.size())) {
        check(cbs_rns_context_create(poly_degree, q.data(), size_q_, p.data(), size_p_, &ctx_), "RnsContext");
    }
    RnsContext(const RnsContext&) = delete;
    RnsContext& operator=(const RnsContext&) = delete;
    ~RnsContext() { cbs_rns_context_destroy(ctx_); }

    [[nodiscard]] cbs_rns_ntt_tables gpu_rns_tables() const {
        cbs_rns_ntt_tables t{};
        check(cbs_rns_context_tables(ctx_, &t), "gpu_rns_tables");
        return t;
    }
    // nwt_2d_radix8_forward_inplace(inout, tables, coeff_modulus_size, start_modulus_idx, stream)
    void nwt_2d_radix8_forward_inplace(uint64_t* inout, size_t coeff_modulus_size, size_t start_modulus_idx,
                                       const cudaStream_t& s) const {
        check(cbs_nwt_2d_radix8_forward_inplace(ctx_, inout, static_cast<uint32_t>(coeff_modulus_size),
                                                static_cast<uint32_t>(start_modulus_idx), as_stream(s)),
              "nwt_2d_radix8_forward_inplace");
    }
    void nwt_2d_radix8_backward_inplace(uint64_t* inout, size_t coeff_modulus_size, size_t start_modulus_idx,
                                        const cudaStream_t& s) const {
        check(cbs_nwt_2d_radix8_backward_inplace(ctx_, inout, static_cast<uint32_t>(coeff_modulus_size),
                                                 static_cast<uint32_t>(start_modulus_idx), as_stream(s)),
              "nwt_2d_radix8_backward_inplace");
    }
    // keyswitch_inplace(context, encrypted, c2, relin_keys, is_relin, stream), CKKS form:
    // ct [count][2][size_ql][N] += keyswitch(c2 [count][size_ql][N]); evks = one key per digit
    void keyswitch_inplace(uint64_t* ct, const uint64_t* c2, const std::vector<const uint64_t*>& evks,
                           uint32_t size_ql, uint32_t count, const cudaStream_t& s) const {
        check(cbs_rns_keyswitch_inplace(ctx_, ct, c2, evks.data(), size_ql, count, as_stream(s)),
              "keyswitch_inplace");
    }
    [[nodiscard]] cbs_rns_context* handle() const { return ctx_; }

   private:
    uint32_t size_q_, size_p_;
    cbs_rns_context* ctx_ = nullptr;
};

}  // namespace cbs_b200
