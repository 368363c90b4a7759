// ref_gpu_rns_shim.cu -- C entry points around the reference's own Phantom RNS tool: a
// PhantomContext built from CKKS EncryptionParameters (include/context.cuh:161) and its
// per-level DRNSTool::modup / moddown_from_NTT (include/rns.cuh:156-164, src/rns_bconv.cu:
// 530-634, 776-828), compiled for sm_100a from the reference sources where they lie by
// `make -C oracle ref_gpu_rns`.  Test infrastructure only: the GPU tests run them beside
// cbs_rns_modup / cbs_rns_moddown_from_ntt on the same data.
#include <cstdint>
#include <vector>

#include "context.cuh"

extern "C" {

// CKKS context over N = 2^log_n with the chain q_all = q_0..q_{size_q-1}, p_0..p_{size_p-1}
// (special primes last, as Phantom's set_special_modulus_size expects); null on failure
void* ref_rns_create(uint32_t log_n, const uint64_t* q_all, uint32_t size_q, uint32_t size_p) {
    try {
        phantom::EncryptionParameters parms(phantom::scheme_type::ckks);
        parms.set_poly_modulus_degree(size_t(1) << log_n);
        std::vector<phantom::arith::Modulus> mods;
        for (uint32_t i = 0; i < size_q + size_p; ++i) mods.emplace_back(q_all[i]);
        parms.set_coeff_modulus(mods);
        parms.set_special_modulus_size(size_p);
        return new PhantomContext(parms);
    } catch (...) {
        return nullptr;
    }
}

void ref_rns_destroy(void* ctx) { delete static_cast<PhantomContext*>(ctx); }

// modup of count polynomials at the level with size_ql primes: c2 [count][size_ql][N] (NTT
// domain) -> dst [count][beta][size_ql + size_p][N]
int ref_rns_modup(void* ctx, uint32_t size_ql, uint64_t* dst, const uint64_t* c2, uint32_t count, void* stream) {
    try {
        auto* c = static_cast<PhantomContext*>(ctx);
        const auto& key = c->get_context_data(0);
        const size_t size_q = key.parms().coeff_modulus().size() - key.parms().special_modulus_size();
        const size_t idx = 1 + (size_q - size_ql);
        const auto& rns = c->get_context_data_rns_tool(idx);
        const size_t n = key.parms().poly_modulus_degree();
        const size_t size_p = key.parms().special_modulus_size();
        const size_t beta = (size_ql + size_p - 1) / size_p;
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        for (uint32_t i = 0; i < count; ++i)
            rns.modup(dst + i * beta * (size_ql + size_p) * n, c2 + i * size_ql * n, c->gpu_rns_tables(),
                      phantom::scheme_type::ckks, s);
        return static_cast<int>(cudaStreamSynchronize(s));
    } catch (...) {
        return -1;
    }
}

// moddown_from_NTT of polys polynomials at the level with size_ql primes: cx
// [polys][size_ql + size_p][N] -> ct [polys][size_ql][N] (added to ct, as the reference does)
int ref_rns_moddown_from_ntt(void* ctx, uint32_t size_ql, uint64_t* ct, uint64_t* cx, uint32_t polys, void* stream) {
    try {
        auto* c = static_cast<PhantomContext*>(ctx);
        const auto& key = c->get_context_data(0);
        const size_t size_q = key.parms().coeff_modulus().size() - key.parms().special_modulus_size();
        const size_t idx = 1 + (size_q - size_ql);
        const auto& rns = c->get_context_data_rns_tool(idx);
        const size_t n = key.parms().poly_modulus_degree();
        const size_t size_p = key.parms().special_modulus_size();
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        for (uint32_t i = 0; i < polys; ++i)
            rns.moddown_from_NTT(ct + i * size_ql * n, cx + i * (size_ql + size_p) * n, c->gpu_rns_tables(),
                                 phantom::scheme_type::ckks, s);
        return static_cast<int>(cudaStreamSynchronize(s));
    } catch (...) {
        return -1;
    }
}

// divide_and_round_q_last_ntt (CKKS rescale_to_next, src/rns.cu:1183-1208) of `size`
// polynomials at the level with size_ql primes: src [size][size_ql][N] (its last limb is
// transformed in place, as in the reference) -> dst [size][size_ql - 1][N]
int ref_rns_rescale(void* ctx, uint32_t size_ql, uint64_t* dst, uint64_t* src, uint32_t size, void* stream) {
    try {
        auto* c = static_cast<PhantomContext*>(ctx);
        const auto& key = c->get_context_data(0);
        const size_t size_q = key.parms().coeff_modulus().size() - key.parms().special_modulus_size();
        const size_t idx = 1 + (size_q - size_ql);
        const auto& rns = c->get_context_data_rns_tool(idx);
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        rns.divide_and_round_q_last_ntt(dst, src, size, c->gpu_rns_tables(), s);
        return static_cast<int>(cudaStreamSynchronize(s));
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
