// cbs_b200.hpp -- header-only C++ facade with the reference's call shapes.
//
// Mirrors the interfaces a caller of the reference binds for this path:
//   * Phantom's 1-D NTT functions (include/ntt.cuh:215-227): same names and argument order,
//     DModulus -> cbs_dmodulus (identical layout), cudaStream_t by const reference;
//   * GPUCirBTSContext (bitwise/include/cirbts/cirbts.cuh:420-498): construction from
//     parameters + max batch, the device-LWE circuit-bootstrapping entry point returning a
//     non-owning DeviceRGSWBatchView, the NTT-table accessors and stream();
//   * the host-input CBS entry points (cirbts.cuh:454-462) on plain LWE / RGSW structs;
//   * Phantom's key-switching types (EncryptionParameters, PhantomContext, PhantomCiphertext,
//     PhantomRelinKey) and keyswitch_inplace (src/eval_key_switch.cu:94), CKKS form;
//   * GPUBinFHEContext::BatchGPUEvalBinGate (bitwise/include/binfhecontext.cuh:53-57).
// Errors surface as exceptions on this side (like OPENFHE_THROW / PHANTOM_CHECK_CUDA in the
// reference); the C ABI underneath never throws.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <map>
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

inline void check_cuda(cudaError_t e, const char* where) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

// Owning device array (the role of phantom::util::cuda_auto_ptr, include/cuda_wrapper.cuh:90):
// grows on resize, contents not preserved.
template <class T>
class DeviceArray {
   public:
    DeviceArray() = default;
    explicit DeviceArray(size_t n) { resize(n); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    DeviceArray(DeviceArray&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr, o.n_ = 0; }
    DeviceArray& operator=(DeviceArray&& o) noexcept {
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        return *this;
    }
    ~DeviceArray() { cudaFree(p_); }
    void resize(size_t n) {
        if (n <= n_) return;
        cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
        check_cuda(cudaMalloc(reinterpret_cast<void**>(&p_), n * sizeof(T)), "DeviceArray");
        n_ = n;
    }
    [[nodiscard]] T* data() const { return p_; }
    [[nodiscard]] size_t size() const { return n_; }

   private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

// The OpenFHE ciphertext types of the reference's CBS and gate interfaces as plain structs:
// an LWE ciphertext (a[n], b mod q; lbcrypto::LWECiphertextImpl) and the host copy of one
// bit's RGSW rows [digitsCC * 2 rows][2 polys][N] (NTT domain; RGSWCiphertext of cirbts.cuh).
struct LWECiphertext {
    std::vector<uint64_t> a;
    uint64_t b = 0;
    uint64_t q = 0;
};
struct RGSWCiphertext {
    std::vector<uint64_t> data;
    uint32_t digitsCC = 0;
    uint32_t N = 0;
};

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

    // The context's CBS backend (the reference reads CIRBTS_BACKEND=ntt|split_fft or
    // CIRBTS_USE_SPLIT_FFT at construction, cirbts-backend.cu:14-38, cirbts-init.cu:333-337):
    // CBS_BR_NTT, CBS_BR_FFT64 or CBS_BR_FFT64_SPLIT (exact, the reference's split_fft)
    void SetBackend(int backend) { check(cbs_context_set_br_backend(ctx_, backend), "SetBackend"); }
    // CIRBTS_PBS_MULTIBIT (cirbts-init.cu:376-386): 1, or 2 / 3 / 4 grouped coefficients per step
    void SetMultibit(uint32_t mb) { check(cbs_context_set_br_multibit(ctx_, mb), "SetMultibit"); }

    // The context's BINFHE_METHOD (GenerateCirBTSContext(paramset, GINX | LMKCDEY),
    // cirbts-init.cu:630-726): CBS_BR_GINX or CBS_BR_LMKCDEY with automorphism keys for 2N - 5 and
    // 5^1 .. 5^numAutoKeys, or the windowed key set (CIRBTS_LMK_AUTOKEYS_WINDOW) when
    // autoKeysWindow > 1; the LMKCDEY keys follow the context's secrets
    void SetMethod(int method, uint32_t numAutoKeys = 10, uint32_t autoKeysWindow = 0) {
        check(cbs_context_set_br_method(ctx_, method, numAutoKeys, autoKeysWindow), "SetMethod");
    }
    // cirbts.cuh:491 LMKCDEY_EvalAcc(params, a, d_acc): a [n] on the host, the masks mod 2N as the
    // bootstrap passes them (negated), d_acc [2][N] on the device (NTT domain), updated in place
    void LMKCDEY_EvalAcc(const std::vector<uint32_t>& a, uint64_t* d_acc) {
        if (a.size() != params_.n)
            throw Error(CBS_ERR_SHAPE_MISMATCH, "LMKCDEY_EvalAcc: a must hold n masks");
        stage_a_.resize(a.size());
        const cudaStream_t s = stream();
        check_cuda(cudaMemcpyAsync(stage_a_.data(), a.data(), a.size() * 4, cudaMemcpyHostToDevice, s), "stage a");
        check(cbs_lmkcdey_eval_acc_batch_device(ctx_, stage_a_.data(), params_.n, d_acc, 1, as_stream(s)),
              "LMKCDEY_EvalAcc");
        check_cuda(cudaStreamSynchronize(s), "LMKCDEY_EvalAcc");  // the staged masks are reused
    }

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

    // cirbts.cuh:462 gpu_CircuitBootstrappingBatchToDevice(params, ek, vector<LWECiphertext>): host
    // LWE ciphertexts staged to the device, then the device-LWE entry point
    [[nodiscard]] DeviceRGSWBatchView gpu_CircuitBootstrappingBatchToDevice(const std::vector<LWECiphertext>& cts) {
        if (cts.empty()) return {};
        const uint32_t n = params_.n, batch = static_cast<uint32_t>(cts.size());
        std::vector<uint64_t> a, b;
        pack(cts, a, b);
        stage_.resize(a.size() + b.size());
        const cudaStream_t s = stream();
        check_cuda(cudaMemcpyAsync(stage_.data(), a.data(), a.size() * 8, cudaMemcpyHostToDevice, s), "stage a");
        check_cuda(cudaMemcpyAsync(stage_.data() + a.size(), b.data(), b.size() * 8, cudaMemcpyHostToDevice, s),
                   "stage b");
        return gpu_CircuitBootstrappingBatchToDeviceFromDeviceLWE(stage_.data(), stage_.data() + a.size(), batch, n);
    }
    // cirbts.cuh:458 gpu_CircuitBootstrappingBatch(params, ek, vector<LWECiphertext>): host RGSWs out
    [[nodiscard]] std::vector<RGSWCiphertext> gpu_CircuitBootstrappingBatch(const std::vector<LWECiphertext>& cts) {
        std::vector<RGSWCiphertext> out;
        if (cts.empty()) return out;
        std::vector<uint64_t> a, b;
        pack(cts, a, b);
        const size_t per = static_cast<size_t>(params_.num_lut) * 4 * params_.N;
        std::vector<uint64_t> rg(per * cts.size());
        check(cbs_circuit_bootstrap_batch(ctx_, a.data(), b.data(), static_cast<uint32_t>(cts.size()), params_.n,
                                          rg.data()),
              "gpu_CircuitBootstrappingBatch");
        out.resize(cts.size());
        for (size_t i = 0; i < cts.size(); ++i) {
            out[i].digitsCC = params_.num_lut;
            out[i].N = params_.N;
            out[i].data.assign(rg.begin() + i * per, rg.begin() + (i + 1) * per);
        }
        return out;
    }
    // cirbts.cuh:454 gpu_CircuitBootstrapping(params, ek, ct)
    [[nodiscard]] RGSWCiphertext gpu_CircuitBootstrapping(const LWECiphertext& ct) {
        return gpu_CircuitBootstrappingBatch(std::vector<LWECiphertext>{ct}).front();
    }

    [[nodiscard]] cbs_context* handle() const { return ctx_; }
    [[nodiscard]] const cbs_params& params() const { return params_; }

   private:
    void pack(const std::vector<LWECiphertext>& cts, std::vector<uint64_t>& a, std::vector<uint64_t>& b) const {
        const uint32_t n = params_.n;
        a.assign(cts.size() * n, 0);
        b.assign(cts.size(), 0);
        for (size_t i = 0; i < cts.size(); ++i) {
            if (cts[i].a.size() != n || cts[i].q != params_.q_lwe)
                throw Error(CBS_ERR_SHAPE_MISMATCH, "LWECiphertext: dimension or modulus differs from the context's");
            std::copy(cts[i].a.begin(), cts[i].a.end(), a.begin() + i * n);
            b[i] = cts[i].b;
        }
    }
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
    DeviceArray<uint64_t> stage_;
    DeviceArray<uint32_t> stage_a_;
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

// ---- Phantom's C++ types for the key-switching path (include/host/encryptionparams.h:37,
//      include/context.cuh:161, include/ciphertext.cuh:8, include/secretkey.h:101,
//      src/eval_key_switch.cu:94) ----
namespace phantom {
// scheme_type of include/host/encryptionparams.h:14 (the key-switching path here is the CKKS form)
enum class scheme_type : std::uint8_t { scheme_none = 0x0, bfv = 0x1, ckks = 0x2, bgv = 0x3 };

// The parameters PhantomContext is built from: ring degree, the key modulus chain (the primes of
// Q followed by the special primes P, as Phantom's coeff_modulus holds them) and the number of
// special primes.  arith::Modulus becomes its value.
class EncryptionParameters {
   public:
    explicit EncryptionParameters(scheme_type scheme = scheme_type::scheme_none) : scheme_(scheme) {}
    void set_poly_modulus_degree(std::size_t n) { poly_modulus_degree_ = n; }
    void set_coeff_modulus(const std::vector<uint64_t>& coeff_modulus) { coeff_modulus_ = coeff_modulus; }
    void set_special_modulus_size(std::size_t size_p) { special_modulus_size_ = size_p; }
    [[nodiscard]] scheme_type scheme() const noexcept { return scheme_; }
    [[nodiscard]] std::size_t poly_modulus_degree() const noexcept { return poly_modulus_degree_; }
    [[nodiscard]] const std::vector<uint64_t>& coeff_modulus() const noexcept { return coeff_modulus_; }
    [[nodiscard]] std::size_t special_modulus_size() const noexcept { return special_modulus_size_; }

   private:
    scheme_type scheme_;
    std::size_t poly_modulus_degree_ = 0;
    std::vector<uint64_t> coeff_modulus_;
    std::size_t special_modulus_size_ = 1;
};
}  // namespace phantom

// PhantomContext: the chain's device tables and the modup / moddown constants.  Chain index c
// (c >= 1) is the level with size_Q - (c - 1) primes of Q, as in Phantom (index 0 = the key level).
class PhantomContext {
   public:
    explicit PhantomContext(const phantom::EncryptionParameters& params)
        : scheme_(params.scheme()), poly_degree_(params.poly_modulus_degree()) {
        if (scheme_ != phantom::scheme_type::ckks)
            throw Error(CBS_ERR_UNSUPPORTED, "PhantomContext: the key-switching path is built for CKKS");
        const auto& chain = params.coeff_modulus();
        const size_t size_p = params.special_modulus_size();
        if (size_p == 0 || chain.size() <= size_p) throw Error(CBS_ERR_INVALID_ARG, "PhantomContext: bad chain");
        q_.assign(chain.begin(), chain.end() - static_cast<std::ptrdiff_t>(size_p));
        p_.assign(chain.end() - static_cast<std::ptrdiff_t>(size_p), chain.end());
        check(cbs_rns_context_create(static_cast<uint32_t>(poly_degree_), q_.data(), static_cast<uint32_t>(q_.size()),
                                     p_.data(), static_cast<uint32_t>(p_.size()), &ctx_),
              "PhantomContext");
        coeff_mod_size_ = chain.size();
    }
    PhantomContext(const PhantomContext&) = delete;
    void operator=(const PhantomContext&) = delete;
    ~PhantomContext() { cbs_rns_context_destroy(ctx_); }

    [[nodiscard]] cbs_rns_ntt_tables gpu_rns_tables() const {
        cbs_rns_ntt_tables t{};
        check(cbs_rns_context_tables(ctx_, &t), "gpu_rns_tables");
        return t;
    }
    // limbs of Q at chain index c
    [[nodiscard]] size_t coeff_modulus_size(size_t chain_index) const {
        if (chain_index < 1 || chain_index > q_.size())
            throw Error(CBS_ERR_INVALID_ARG, "PhantomContext: chain index out of range");
        return q_.size() - (chain_index - 1);
    }
    [[nodiscard]] phantom::scheme_type scheme() const { return scheme_; }
    [[nodiscard]] size_t poly_degree() const { return poly_degree_; }
    [[nodiscard]] size_t coeff_mod_size() const { return coeff_mod_size_; }
    [[nodiscard]] size_t special_modulus_size() const { return p_.size(); }
    [[nodiscard]] cbs_rns_context* handle() const { return ctx_; }

   private:
    phantom::scheme_type scheme_;
    size_t poly_degree_ = 0, coeff_mod_size_ = 0;
    std::vector<uint64_t> q_, p_;
    cbs_rns_context* ctx_ = nullptr;
};

// PhantomCiphertext: size polynomials of coeff_modulus_size limbs, NTT form, device resident
// ([size][coeff_modulus_size][N] words).
class PhantomCiphertext {
   public:
    PhantomCiphertext() = default;
    void resize(const PhantomContext& context, size_t chain_index, size_t size, const cudaStream_t&) {
        chain_index_ = chain_index;
        size_ = size;
        coeff_modulus_size_ = context.coeff_modulus_size(chain_index);
        poly_modulus_degree_ = context.poly_degree();
        data_.resize(size_ * coeff_modulus_size_ * poly_modulus_degree_);
    }
    [[nodiscard]] uint64_t* data() const { return data_.data(); }
    [[nodiscard]] size_t size() const { return size_; }
    [[nodiscard]] size_t chain_index() const { return chain_index_; }
    [[nodiscard]] size_t coeff_modulus_size() const { return coeff_modulus_size_; }
    [[nodiscard]] size_t poly_modulus_degree() const { return poly_modulus_degree_; }
    [[nodiscard]] bool is_ntt_form() const { return is_ntt_form_; }
    // CKKS scale bookkeeping (PhantomCiphertext::GetScalingFactor / SetScalingFactor)
    [[nodiscard]] double GetScalingFactor() const { return scale_; }
    void SetScalingFactor(double scale) { scale_ = scale; }
    // keep the first min(size, new_size) polynomials, grow or shrink to new_size (device copy)
    void resize_keep(size_t new_size, const cudaStream_t& stream) {
        const size_t per = coeff_modulus_size_ * poly_modulus_degree_;
        if (new_size > size_) {
            DeviceArray<uint64_t> bigger(new_size * per);
            check_cuda(cudaMemcpyAsync(bigger.data(), data_.data(), size_ * per * 8, cudaMemcpyDeviceToDevice, stream),
                       "PhantomCiphertext");
            data_ = std::move(bigger);
        }
        size_ = new_size;
    }
    // the storage of a ciphertext one level down (chain index + 1), same size
    void reset_level(const PhantomContext& context, size_t chain_index, DeviceArray<uint64_t>&& data) {
        chain_index_ = chain_index;
        coeff_modulus_size_ = context.coeff_modulus_size(chain_index);
        data_ = std::move(data);
    }

   private:
    size_t size_ = 0, chain_index_ = 0, coeff_modulus_size_ = 0, poly_modulus_degree_ = 0;
    bool is_ntt_form_ = true;
    double scale_ = 1.0;
    DeviceArray<uint64_t> data_;
};

// PhantomPlaintext: one NTT-form polynomial of coeff_modulus_size limbs on the device
// ([coeff_modulus_size][N] words) at chain index c.
class PhantomPlaintext {
   public:
    PhantomPlaintext() = default;
    void resize(const PhantomContext& context, size_t chain_index) {
        chain_index_ = chain_index;
        coeff_modulus_size_ = context.coeff_modulus_size(chain_index);
        data_.resize(coeff_modulus_size_ * context.poly_degree());
    }
    [[nodiscard]] uint64_t* data() const { return data_.data(); }
    [[nodiscard]] size_t chain_index() const { return chain_index_; }
    [[nodiscard]] size_t coeff_modulus_size() const { return coeff_modulus_size_; }

   private:
    size_t chain_index_ = 0, coeff_modulus_size_ = 0;
    DeviceArray<uint64_t> data_;
};

// PhantomRelinKey: beta switching keys, one per digit, each [2][size_Q + size_P][N] on the device;
// public_keys_ptr() lists them (host array of device pointers here, a device array in Phantom).
class PhantomRelinKey {
   public:
    PhantomRelinKey() = default;
    // host keys [beta][2][size_Q + size_P][N], uploaded
    PhantomRelinKey(const PhantomContext& context, const std::vector<uint64_t>& keys, size_t beta) {
        const size_t per = 2 * context.coeff_mod_size() * context.poly_degree();
        if (keys.size() != beta * per) throw Error(CBS_ERR_SHAPE_MISMATCH, "PhantomRelinKey: key size");
        data_.resize(keys.size());
        check_cuda(cudaMemcpy(data_.data(), keys.data(), keys.size() * 8, cudaMemcpyHostToDevice), "PhantomRelinKey");
        for (size_t b = 0; b < beta; ++b) ptrs_.push_back(data_.data() + b * per);
    }
    PhantomRelinKey(const PhantomRelinKey&) = delete;
    PhantomRelinKey& operator=(const PhantomRelinKey&) = delete;
    PhantomRelinKey(PhantomRelinKey&&) = default;
    PhantomRelinKey& operator=(PhantomRelinKey&&) = default;
    [[nodiscard]] const uint64_t* const* public_keys_ptr() const { return ptrs_.data(); }
    [[nodiscard]] size_t dnum() const { return ptrs_.size(); }

   private:
    DeviceArray<uint64_t> data_;
    std::vector<const uint64_t*> ptrs_;
};

// keyswitch_inplace (src/eval_key_switch.cu:94-181), CKKS: encrypted (size >= 2 polys at chain
// index c, size_Ql = its coeff_modulus_size limbs) += keyswitch(c2 [size_Ql][N]) with the relin
// keys' digits; is_relin only changes the reference's BFV level choice and is accepted for shape.
inline void keyswitch_inplace(const PhantomContext& context, PhantomCiphertext& encrypted, uint64_t* c2,
                              const PhantomRelinKey& relin_keys, bool is_relin, const cudaStream_t& stream) {
    (void)is_relin;
    if (context.scheme() != phantom::scheme_type::ckks)
        throw Error(CBS_ERR_UNSUPPORTED, "keyswitch_inplace: unsupported scheme in keyswitch_inplace");
    const uint32_t size_ql = static_cast<uint32_t>(encrypted.coeff_modulus_size());
    check(cbs_rns_keyswitch_inplace(context.handle(), encrypted.data(), c2, relin_keys.public_keys_ptr(), size_ql, 1,
                                    as_stream(stream)),
          "keyswitch_inplace");
}

// ---- CKKS evaluator (include/evaluate.cuh; csrc/ckks.cu), NTT-form ciphertexts ----
inline uint32_t level_limbs(const PhantomCiphertext& ct) { return static_cast<uint32_t>(ct.coeff_modulus_size()); }
inline void same_level(const PhantomCiphertext& a, const PhantomCiphertext& b, const char* what) {
    if (a.chain_index() != b.chain_index()) throw Error(CBS_ERR_SHAPE_MISMATCH, std::string(what) + ": level mismatch");
}

// add_inplace (include/evaluate.cuh:46)
inline void add_inplace(const PhantomContext& context, PhantomCiphertext& encrypted1,
                        const PhantomCiphertext& encrypted2) {
    same_level(encrypted1, encrypted2, "add_inplace");
    if (encrypted1.size() != encrypted2.size()) throw Error(CBS_ERR_SHAPE_MISMATCH, "add_inplace: size mismatch");
    check(cbs_ckks_add_inplace(context.handle(), encrypted1.data(), encrypted2.data(),
                               static_cast<uint32_t>(encrypted1.size()), level_limbs(encrypted1), nullptr),
          "add_inplace");
}
// sub_inplace (include/evaluate.cuh:61): encrypted1 -= encrypted2, or encrypted2 - encrypted1
inline void sub_inplace(const PhantomContext& context, PhantomCiphertext& encrypted1,
                        const PhantomCiphertext& encrypted2, bool negate = false) {
    same_level(encrypted1, encrypted2, "sub_inplace");
    if (encrypted1.size() != encrypted2.size()) throw Error(CBS_ERR_SHAPE_MISMATCH, "sub_inplace: size mismatch");
    check(cbs_ckks_sub_inplace(context.handle(), encrypted1.data(), encrypted2.data(),
                               static_cast<uint32_t>(encrypted1.size()), level_limbs(encrypted1), negate ? 1 : 0,
                               nullptr),
          "sub_inplace");
}
// negate_inplace (include/evaluate.cuh:37)
inline void negate_inplace(const PhantomContext& context, PhantomCiphertext& encrypted) {
    check(cbs_ckks_negate_inplace(context.handle(), encrypted.data(), static_cast<uint32_t>(encrypted.size()),
                                  level_limbs(encrypted), nullptr),
          "negate_inplace");
}
// multiply_plain_inplace (include/evaluate.cuh:94)
inline void multiply_plain_inplace(const PhantomContext& context, PhantomCiphertext& encrypted,
                                   const PhantomPlaintext& plain) {
    if (plain.chain_index() != encrypted.chain_index())
        throw Error(CBS_ERR_SHAPE_MISMATCH, "multiply_plain_inplace: level mismatch");
    check(cbs_ckks_multiply_plain_inplace(context.handle(), encrypted.data(), plain.data(),
                                          static_cast<uint32_t>(encrypted.size()), level_limbs(encrypted), nullptr),
          "multiply_plain_inplace");
}
// multiply_inplace (include/evaluate.cuh:105): size-2 operands, encrypted1 becomes size 3;
// CKKS scales multiply
inline void multiply_inplace(const PhantomContext& context, PhantomCiphertext& encrypted1,
                             const PhantomCiphertext& encrypted2) {
    same_level(encrypted1, encrypted2, "multiply_inplace");
    if (encrypted1.size() != 2 || encrypted2.size() != 2)
        throw Error(CBS_ERR_UNSUPPORTED, "multiply_inplace: size-2 ciphertexts");
    const bool square = &encrypted1 == &encrypted2;
    encrypted1.resize_keep(3, cudaStream_t{});
    check(cbs_ckks_multiply_inplace(context.handle(), encrypted1.data(), square ? encrypted1.data() : encrypted2.data(),
                                    level_limbs(encrypted1), nullptr),
          "multiply_inplace");
    encrypted1.SetScalingFactor(encrypted1.GetScalingFactor() * encrypted2.GetScalingFactor());
}
// relinearize_inplace (include/evaluate.cuh:125)
inline void relinearize_inplace(const PhantomContext& context, PhantomCiphertext& encrypted,
                                const PhantomRelinKey& relin_keys) {
    if (encrypted.size() != 3) throw Error(CBS_ERR_UNSUPPORTED, "relinearize_inplace: destination_size must be 3");
    check(cbs_ckks_relinearize_inplace(context.handle(), encrypted.data(), relin_keys.public_keys_ptr(),
                                       level_limbs(encrypted), nullptr),
          "relinearize_inplace");
    encrypted.resize_keep(2, cudaStream_t{});
}
// multiply_and_relin_inplace (include/evaluate.cuh:115)
inline void multiply_and_relin_inplace(const PhantomContext& context, PhantomCiphertext& encrypted1,
                                       const PhantomCiphertext& encrypted2, const PhantomRelinKey& relin_keys) {
    multiply_inplace(context, encrypted1, encrypted2);
    relinearize_inplace(context, encrypted1, relin_keys);
}
// rescale_to_next_inplace (include/evaluate.cuh:140): one level down, the scale divided by the
// dropped prime
inline void rescale_to_next_inplace(const PhantomContext& context, PhantomCiphertext& encrypted, double q_last) {
    const size_t next = encrypted.chain_index() + 1;
    const uint32_t limbs = level_limbs(encrypted);
    DeviceArray<uint64_t> out(encrypted.size() * (limbs - 1) * context.poly_degree());
    check(cbs_ckks_rescale_to_next(context.handle(), out.data(), encrypted.data(),
                                   static_cast<uint32_t>(encrypted.size()), limbs, nullptr),
          "rescale_to_next");
    encrypted.reset_level(context, next, std::move(out));
    encrypted.SetScalingFactor(encrypted.GetScalingFactor() / q_last);
}
// mod_switch_to_next_inplace (include/evaluate.cuh:149), CKKS: the last limb dropped
inline void mod_switch_to_next_inplace(const PhantomContext& context, PhantomCiphertext& encrypted) {
    const size_t next = encrypted.chain_index() + 1;
    const uint32_t limbs = level_limbs(encrypted);
    DeviceArray<uint64_t> out(encrypted.size() * (limbs - 1) * context.poly_degree());
    check(cbs_ckks_mod_switch_to_next(context.handle(), out.data(), encrypted.data(),
                                      static_cast<uint32_t>(encrypted.size()), limbs, nullptr),
          "mod_switch_to_next");
    encrypted.reset_level(context, next, std::move(out));
}

// PhantomGaloisKey: one switching key (PhantomRelinKey shape) per Galois element
class PhantomGaloisKey {
   public:
    void insert(uint32_t galois_elt, PhantomRelinKey&& key) { keys_[galois_elt] = std::move(key); }
    [[nodiscard]] const PhantomRelinKey& get_relin_keys(uint32_t galois_elt) const {
        auto it = keys_.find(galois_elt);
        if (it == keys_.end()) throw Error(CBS_ERR_INVALID_ARG, "PhantomGaloisKey: no key for this Galois element");
        return it->second;
    }

   private:
    std::map<uint32_t, PhantomRelinKey> keys_;
};

// apply_galois_inplace (include/evaluate.cuh:215) and rotate_inplace (:229), CKKS
inline void apply_galois_inplace(const PhantomContext& context, PhantomCiphertext& encrypted, uint32_t galois_elt,
                                 const PhantomGaloisKey& galois_keys) {
    if (encrypted.size() != 2) throw Error(CBS_ERR_UNSUPPORTED, "apply_galois_inplace: encrypted size must be 2");
    check(cbs_ckks_apply_galois_inplace(context.handle(), encrypted.data(), galois_elt,
                                        galois_keys.get_relin_keys(galois_elt).public_keys_ptr(),
                                        level_limbs(encrypted), nullptr),
          "apply_galois_inplace");
}
inline void rotate_inplace(const PhantomContext& context, PhantomCiphertext& encrypted, int step,
                           const PhantomGaloisKey& galois_keys) {
    const uint32_t elt = cbs_ckks_galois_elt_from_step(step, static_cast<uint32_t>(context.poly_degree()));
    if (!elt) throw Error(CBS_ERR_INVALID_ARG, "rotate_inplace: step count too large");
    apply_galois_inplace(context, encrypted, elt, galois_keys);
}

// ---- GPUBinFHEContext (bitwise/include/binfhecontext.cuh:8-118): gate bootstrapping on the
//      32-bit torus (LWECiphertext::q = 2^32) ----
enum BINGATE { OR = CBS_GATE_OR, AND = CBS_GATE_AND, NOR = CBS_GATE_NOR, NAND = CBS_GATE_NAND, XOR = CBS_GATE_XOR,
               XNOR = CBS_GATE_XNOR };

class GPUBinFHEContext {
   public:
    explicit GPUBinFHEContext(const cbs_gate_params& params, uint32_t max_batch = 1024)
        : params_(params), max_batch_(max_batch) {
        check(cbs_gate_context_create(&params_, max_batch_, &ctx_), "GPUBinFHEContext");
    }
    GPUBinFHEContext(const GPUBinFHEContext&) = delete;
    GPUBinFHEContext& operator=(const GPUBinFHEContext&) = delete;
    ~GPUBinFHEContext() { cbs_gate_context_destroy(ctx_); }

    // GPUBTKeyGen (binfhecontext.cuh:38), from a seed
    void GPUBTKeyGen(uint64_t seed) { check(cbs_gate_keygen(ctx_, seed), "GPUBTKeyGen"); }

    // binfhecontext.cuh:53-57
    [[nodiscard]] std::vector<LWECiphertext> BatchGPUEvalBinGate(BINGATE gate, const std::vector<LWECiphertext>& v_ct1,
                                                                 const std::vector<LWECiphertext>& v_ct2,
                                                                 const cudaStream_t& stream = nullptr) {
        if (v_ct1.size() != v_ct2.size()) throw Error(CBS_ERR_SHAPE_MISMATCH, "BatchGPUEvalBinGate: batch sizes");
        const size_t count = v_ct1.size(), n = params_.n;
        std::vector<LWECiphertext> out(count);
        if (!count) return out;
        if (count > max_batch_) throw Error(CBS_ERR_SHAPE_MISMATCH, "BatchGPUEvalBinGate: batch above max_batch");
        std::vector<uint32_t> a1(count * n), b1(count), a2(count * n), b2(count);
        auto put = [&](const std::vector<LWECiphertext>& v, std::vector<uint32_t>& a, std::vector<uint32_t>& b) {
            for (size_t i = 0; i < count; ++i) {
                if (v[i].a.size() != n || v[i].q != (uint64_t(1) << 32))
                    throw Error(CBS_ERR_SHAPE_MISMATCH, "BatchGPUEvalBinGate: dimension or modulus");
                for (size_t j = 0; j < n; ++j) a[i * n + j] = static_cast<uint32_t>(v[i].a[j]);
                b[i] = static_cast<uint32_t>(v[i].b);
            }
        };
        put(v_ct1, a1, b1);
        put(v_ct2, a2, b2);
        const size_t words = 3 * (count * n + count);  // in1, in2, out
        dev_.resize(words);
        uint32_t* d = dev_.data();
        uint32_t *da1 = d, *db1 = da1 + count * n, *da2 = db1 + count, *db2 = da2 + count * n, *doa = db2 + count,
                 *dob = doa + count * n;
        check_cuda(cudaMemcpyAsync(da1, a1.data(), a1.size() * 4, cudaMemcpyHostToDevice, stream), "in1 a");
        check_cuda(cudaMemcpyAsync(db1, b1.data(), b1.size() * 4, cudaMemcpyHostToDevice, stream), "in1 b");
        check_cuda(cudaMemcpyAsync(da2, a2.data(), a2.size() * 4, cudaMemcpyHostToDevice, stream), "in2 a");
        check_cuda(cudaMemcpyAsync(db2, b2.data(), b2.size() * 4, cudaMemcpyHostToDevice, stream), "in2 b");
        check(cbs_gate_eval_batch_device(ctx_, static_cast<int>(gate), da1, db1, da2, db2, static_cast<uint32_t>(count),
                                         doa, dob, as_stream(stream)),
              "BatchGPUEvalBinGate");
        std::vector<uint32_t> oa(count * n), ob(count);
        check_cuda(cudaMemcpyAsync(oa.data(), doa, oa.size() * 4, cudaMemcpyDeviceToHost, stream), "out a");
        check_cuda(cudaMemcpyAsync(ob.data(), dob, ob.size() * 4, cudaMemcpyDeviceToHost, stream), "out b");
        check_cuda(cudaStreamSynchronize(stream), "BatchGPUEvalBinGate");
        for (size_t i = 0; i < count; ++i) {
            out[i].a.assign(oa.begin() + i * n, oa.begin() + (i + 1) * n);
            out[i].b = ob[i];
            out[i].q = uint64_t(1) << 32;
        }
        return out;
    }

    // The functional evaluators (binfhecontext.cuh:60-118; binfhe-base-scheme-batch.cu:366-712).
    // Their LWECiphertexts carry a power-of-two modulus q; the parameter set's LWE modulus and the
    // error bound beta (the reference's Getq() and GetBeta()) are set here (defaults N and 128).
    void SetFunctionalParams(uint32_t lweModulus, uint32_t beta) {
        lwe_q_ = lweModulus;
        beta_ = beta;
    }
    // GPUEvalFunc / BatchGPUEvalFunc: LUT [q] over Z_q, q the ciphertexts' modulus
    [[nodiscard]] std::vector<LWECiphertext> BatchGPUEvalFunc(const std::vector<LWECiphertext>& v_ct,
                                                              const std::vector<uint64_t>& LUT,
                                                              const cudaStream_t& stream = nullptr) {
        const uint64_t q = common_modulus(v_ct, "BatchGPUEvalFunc");
        if (LUT.size() != q) throw Error(CBS_ERR_SHAPE_MISMATCH, "BatchGPUEvalFunc: the LUT must have q entries");
        std::vector<uint32_t> lut(LUT.begin(), LUT.end());
        return unary(v_ct, q, stream, [&](const uint32_t* a, const uint32_t* b, uint32_t count, uint32_t* oa,
                                          uint32_t* ob, cbs_stream_t s) {
            return cbs_gate_eval_func_batch_device(ctx_, a, b, count, static_cast<uint32_t>(q), lut.data(), beta_, oa,
                                                   ob, s);
        });
    }
    [[nodiscard]] LWECiphertext GPUEvalFunc(const LWECiphertext& ct, const std::vector<uint64_t>& LUT,
                                            const cudaStream_t& stream = nullptr) {
        return BatchGPUEvalFunc(std::vector<LWECiphertext>{ct}, LUT, stream).front();
    }
    // GPUEvalFloor / BatchGPUEvalFloor
    [[nodiscard]] std::vector<LWECiphertext> BatchGPUEvalFloor(const std::vector<LWECiphertext>& v_ct,
                                                               uint32_t roundbits = 0,
                                                               const cudaStream_t& stream = nullptr) {
        const uint64_t mod = common_modulus(v_ct, "BatchGPUEvalFloor");
        return unary(v_ct, mod, stream, [&](const uint32_t* a, const uint32_t* b, uint32_t count, uint32_t* oa,
                                            uint32_t* ob, cbs_stream_t s) {
            return cbs_gate_eval_floor_batch_device(ctx_, a, b, count, mod, lwe_q(), roundbits, beta_, oa, ob, s);
        });
    }
    [[nodiscard]] LWECiphertext GPUEvalFloor(const LWECiphertext& ct, uint32_t roundbits = 0,
                                             const cudaStream_t& stream = nullptr) {
        return BatchGPUEvalFloor(std::vector<LWECiphertext>{ct}, roundbits, stream).front();
    }
    // GPUEvalSign / BatchGPUEvalSign: outputs modulo the LWE modulus
    [[nodiscard]] std::vector<LWECiphertext> BatchGPUEvalSign(const std::vector<LWECiphertext>& v_ct,
                                                              bool schemeSwitch = false,
                                                              const cudaStream_t& stream = nullptr) {
        const uint64_t mod = common_modulus(v_ct, "BatchGPUEvalSign");
        return unary(v_ct, lwe_q(), stream, [&](const uint32_t* a, const uint32_t* b, uint32_t count, uint32_t* oa,
                                                uint32_t* ob, cbs_stream_t s) {
            return cbs_gate_eval_sign_batch_device(ctx_, a, b, count, mod, lwe_q(), beta_, schemeSwitch ? 1 : 0, oa, ob,
                                                   s);
        });
    }
    [[nodiscard]] LWECiphertext GPUEvalSign(const LWECiphertext& ct, bool schemeSwitch = false,
                                            const cudaStream_t& stream = nullptr) {
        return BatchGPUEvalSign(std::vector<LWECiphertext>{ct}, schemeSwitch, stream).front();
    }
    // GPUEvalDecomp / BatchGPUEvalDecomp: per ciphertext its digits, least significant first
    [[nodiscard]] std::vector<std::vector<LWECiphertext>> BatchGPUEvalDecomp(const std::vector<LWECiphertext>& v_ct,
                                                                             const cudaStream_t& stream = nullptr) {
        const uint64_t mod = common_modulus(v_ct, "BatchGPUEvalDecomp");
        const size_t count = v_ct.size(), n = params_.n;
        std::vector<std::vector<LWECiphertext>> out(count);
        if (!count) return out;
        uint32_t digits = 0;  // ask for the digit count first
        const uint32_t q = lwe_q();
        (void)cbs_gate_eval_decomp_batch_device(ctx_, nullptr, nullptr, 0, mod, q, beta_, nullptr, nullptr, &digits,
                                                nullptr);
        if (digits == 0) throw Error(CBS_ERR_INVALID_ARG, std::string("BatchGPUEvalDecomp: ") + cbs_last_error());
        upload(v_ct, stream);
        uint32_t* d = dev_.data();
        const size_t in_words = count * n + count;
        dev_out_.resize(digits * in_words);
        uint32_t *oa = dev_out_.data(), *ob = oa + digits * count * n;
        uint32_t cap = digits;
        check(cbs_gate_eval_decomp_batch_device(ctx_, d, d + count * n, static_cast<uint32_t>(count), mod, q, beta_,
                                                oa, ob, &cap, as_stream(stream)),
              "BatchGPUEvalDecomp");
        std::vector<uint32_t> ha(digits * count * n), hb(digits * count);
        check_cuda(cudaMemcpyAsync(ha.data(), oa, ha.size() * 4, cudaMemcpyDeviceToHost, stream), "digits a");
        check_cuda(cudaMemcpyAsync(hb.data(), ob, hb.size() * 4, cudaMemcpyDeviceToHost, stream), "digits b");
        check_cuda(cudaStreamSynchronize(stream), "BatchGPUEvalDecomp");
        // digit moduli: q for every floor, the final modulus for the last
        const int qb = log2_of(q), bb = log2_of(beta_);
        int mb = log2_of(mod);
        std::vector<uint64_t> mods;
        while (mb > qb) {
            mods.push_back(q);
            mb = mb - qb + 1 + bb;
        }
        mods.push_back(uint64_t(1) << mb);
        for (size_t i = 0; i < count; ++i)
            for (uint32_t k = 0; k < digits; ++k) {
                LWECiphertext c;
                c.a.assign(ha.begin() + (k * count + i) * n, ha.begin() + (k * count + i + 1) * n);
                c.b = hb[k * count + i];
                c.q = mods[k];
                out[i].push_back(std::move(c));
            }
        return out;
    }
    [[nodiscard]] std::vector<LWECiphertext> GPUEvalDecomp(const LWECiphertext& ct, const cudaStream_t& stream = nullptr) {
        return BatchGPUEvalDecomp(std::vector<LWECiphertext>{ct}, stream).front();
    }

    [[nodiscard]] cbs_gate_context* handle() const { return ctx_; }
    [[nodiscard]] const cbs_gate_params& params() const { return params_; }

   private:
    static int log2_of(uint64_t v) {
        int b = 0;
        while ((uint64_t(1) << b) < v) ++b;
        return b;
    }
    uint32_t lwe_q() const { return lwe_q_ ? lwe_q_ : params_.N; }
    uint64_t common_modulus(const std::vector<LWECiphertext>& v, const char* who) const {
        if (v.empty()) return lwe_q();
        const uint64_t q = v[0].q;
        for (const auto& c : v)
            if (c.q != q || c.a.size() != params_.n)
                throw Error(CBS_ERR_SHAPE_MISMATCH, std::string(who) + ": ciphertexts of one modulus and dimension n");
        if (v.size() > max_batch_) throw Error(CBS_ERR_SHAPE_MISMATCH, std::string(who) + ": batch above max_batch");
        return q;
    }
    void upload(const std::vector<LWECiphertext>& v, const cudaStream_t& stream) {
        const size_t count = v.size(), n = params_.n;
        std::vector<uint32_t> h(count * n + count);
        for (size_t i = 0; i < count; ++i) {
            for (size_t j = 0; j < n; ++j) h[i * n + j] = static_cast<uint32_t>(v[i].a[j]);
            h[count * n + i] = static_cast<uint32_t>(v[i].b);
        }
        dev_.resize(h.size());
        check_cuda(cudaMemcpyAsync(dev_.data(), h.data(), h.size() * 4, cudaMemcpyHostToDevice, stream), "upload");
        check_cuda(cudaStreamSynchronize(stream), "upload");  // h is a temporary
    }
    template <class F>
    std::vector<LWECiphertext> unary(const std::vector<LWECiphertext>& v, uint64_t out_q, const cudaStream_t& stream,
                                     F fn) {
        const size_t count = v.size(), n = params_.n;
        std::vector<LWECiphertext> out(count);
        if (!count) return out;
        upload(v, stream);
        dev_out_.resize(count * n + count);
        uint32_t *d = dev_.data(), *o = dev_out_.data();
        check(fn(d, d + count * n, static_cast<uint32_t>(count), o, o + count * n, as_stream(stream)), "evaluator");
        std::vector<uint32_t> h(count * n + count);
        check_cuda(cudaMemcpyAsync(h.data(), o, h.size() * 4, cudaMemcpyDeviceToHost, stream), "download");
        check_cuda(cudaStreamSynchronize(stream), "evaluator");
        for (size_t i = 0; i < count; ++i) {
            out[i].a.assign(h.begin() + i * n, h.begin() + (i + 1) * n);
            out[i].b = h[count * n + i];
            out[i].q = out_q;
        }
        return out;
    }
    cbs_gate_params params_;
    uint32_t max_batch_;
    cbs_gate_context* ctx_ = nullptr;
    DeviceArray<uint32_t> dev_, dev_out_;
    uint32_t lwe_q_ = 0, beta_ = 128;
};

}  // namespace cbs_b200
