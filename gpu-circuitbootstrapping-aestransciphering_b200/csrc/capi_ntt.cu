// capi_ntt.cu -- C ABI: status/error plumbing and the Phantom 1-D NTT entry points.
#include <cstring>
#include <string>

#include "common.cuh"
#include "host_math.h"

namespace cbs {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

cudaError_t ntt_forward(uint64_t* out, const uint64_t* in, const uint64_t* tw, const uint64_t* tws,
                        const cbs_dmodulus* mod, size_t dim, size_t batch, cudaStream_t s);
cudaError_t ntt_inverse(uint64_t* out, const uint64_t* in, const uint32_t* map, const uint64_t* itw,
                        const uint64_t* itws, const cbs_dmodulus* mod, const uint64_t* sc, const uint64_t* scs,
                        size_t dim, size_t batch, cudaStream_t s);

static bool dim_ok(size_t dim) { return dim == 1024 || dim == 2048 || dim == 4096; }

}  // namespace cbs

using namespace cbs;

extern "C" {

const char* cbs_last_error(void) { return g_last_error.c_str(); }

int cbs_abi_version(void) { return 1; }

cbs_status cbs_fnwt_1d_opt_batched(uint64_t* d_inout, const uint64_t* d_twiddles, const uint64_t* d_twiddles_shoup,
                                   const cbs_dmodulus* d_modulus, size_t dim, size_t batch, cbs_stream_t stream) {
    return cbs_fnwt_1d_opt_outofplace_batched(d_inout, d_inout, d_twiddles, d_twiddles_shoup, d_modulus, dim, batch,
                                              stream);
}

cbs_status cbs_fnwt_1d_opt_outofplace_batched(uint64_t* d_out, const uint64_t* d_in, const uint64_t* d_twiddles,
                                              const uint64_t* d_twiddles_shoup, const cbs_dmodulus* d_modulus,
                                              size_t dim, size_t batch, cbs_stream_t stream) {
    CBS_CHECK_ARG(dim_ok(dim), "fnwt: dim must be 1024, 2048 or 4096");
    if (batch == 0) return CBS_OK;
    CBS_CHECK_ARG(d_out && d_in && d_twiddles && d_twiddles_shoup && d_modulus, "fnwt: null pointer");
    CBS_CHECK_ARG(batch <= 0x7fffffffu, "fnwt: batch too large");
    CBS_CUDA_TRY(ntt_forward(d_out, d_in, d_twiddles, d_twiddles_shoup, d_modulus, dim, batch,
                             reinterpret_cast<cudaStream_t>(stream)));
    return CBS_OK;
}

cbs_status cbs_inwt_1d_opt_batched(uint64_t* d_inout, const uint64_t* d_itwiddles, const uint64_t* d_itwiddles_shoup,
                                   const cbs_dmodulus* d_modulus, const uint64_t* d_scalar,
                                   const uint64_t* d_scalar_shoup, size_t dim, size_t batch, cbs_stream_t stream) {
    return cbs_inwt_1d_opt_outofplace_batched(d_inout, d_inout, d_itwiddles, d_itwiddles_shoup, d_modulus, d_scalar,
                                              d_scalar_shoup, dim, batch, stream);
}

cbs_status cbs_inwt_1d_opt_outofplace_batched(uint64_t* d_out, const uint64_t* d_in, const uint64_t* d_itwiddles,
                                              const uint64_t* d_itwiddles_shoup, const cbs_dmodulus* d_modulus,
                                              const uint64_t* d_scalar, const uint64_t* d_scalar_shoup, size_t dim,
                                              size_t batch, cbs_stream_t stream) {
    CBS_CHECK_ARG(dim_ok(dim), "inwt: dim must be 1024, 2048 or 4096");
    if (batch == 0) return CBS_OK;
    CBS_CHECK_ARG(d_out && d_in && d_itwiddles && d_itwiddles_shoup && d_modulus && d_scalar && d_scalar_shoup,
                  "inwt: null pointer");
    CBS_CHECK_ARG(batch <= 0x7fffffffu, "inwt: batch too large");
    CBS_CUDA_TRY(ntt_inverse(d_out, d_in, nullptr, d_itwiddles, d_itwiddles_shoup, d_modulus, d_scalar,
                             d_scalar_shoup, dim, batch, reinterpret_cast<cudaStream_t>(stream)));
    return CBS_OK;
}

cbs_status cbs_inwt_1d_opt_permute_batched(uint64_t* d_out, const uint64_t* d_in, const uint32_t* d_map,
                                           const uint64_t* d_itwiddles, const uint64_t* d_itwiddles_shoup,
                                           const cbs_dmodulus* d_modulus, const uint64_t* d_scalar,
                                           const uint64_t* d_scalar_shoup, size_t dim, size_t batch,
                                           cbs_stream_t stream) {
    CBS_CHECK_ARG(dim_ok(dim), "inwt_permute: dim must be 1024, 2048 or 4096");
    if (batch == 0) return CBS_OK;
    CBS_CHECK_ARG(d_out && d_in && d_map && d_itwiddles && d_itwiddles_shoup && d_modulus && d_scalar &&
                      d_scalar_shoup,
                  "inwt_permute: null pointer");
    CBS_CHECK_ARG(d_out != d_in, "inwt_permute: in-place permutation is not supported");
    CBS_CHECK_ARG(batch <= 0x7fffffffu, "inwt_permute: batch too large");
    CBS_CUDA_TRY(ntt_inverse(d_out, d_in, d_map, d_itwiddles, d_itwiddles_shoup, d_modulus, d_scalar, d_scalar_shoup,
                             dim, batch, reinterpret_cast<cudaStream_t>(stream)));
    return CBS_OK;
}

cbs_status cbs_ntt_tables_host(uint32_t dim, uint64_t q, uint64_t* h_twiddles, uint64_t* h_twiddles_shoup,
                               uint64_t* h_itwiddles, uint64_t* h_itwiddles_shoup, uint64_t* h_n_inv,
                               cbs_dmodulus* h_modulus) {
    CBS_CHECK_ARG(dim >= 2 && (dim & (dim - 1)) == 0, "ntt_tables: dim must be a power of two");
    CBS_CHECK_ARG(q > 2 && q < (1ull << 62), "ntt_tables: q out of range");
    host::NttTables t;
    if (!host::make_ntt_tables(dim, q, t)) {
        set_error("ntt_tables: q is not an NTT-friendly prime for this dim");
        return CBS_ERR_INVALID_ARG;
    }
    const size_t bytes = size_t(dim) * 8;
    if (h_twiddles) std::memcpy(h_twiddles, t.rp.data(), bytes);
    if (h_twiddles_shoup) std::memcpy(h_twiddles_shoup, t.rp_sh.data(), bytes);
    if (h_itwiddles) std::memcpy(h_itwiddles, t.irp.data(), bytes);
    if (h_itwiddles_shoup) std::memcpy(h_itwiddles_shoup, t.irp_sh.data(), bytes);
    if (h_n_inv) {
        h_n_inv[0] = t.n_inv;
        h_n_inv[1] = t.n_inv_sh;
    }
    if (h_modulus) {
        h_modulus->value = q;
        h_modulus->const_ratio[0] = t.ratio0;
        h_modulus->const_ratio[1] = t.ratio1;
    }
    return CBS_OK;
}

cbs_status cbs_get_primes(uint32_t ntt_size, int bit_size, uint32_t count, uint64_t* h_out) {
    CBS_CHECK_ARG(h_out || count == 0, "get_primes: null output");
    std::vector<uint64_t> v;
    if (!host::get_primes(ntt_size, bit_size, count, v)) {
        set_error("get_primes: failed to find enough qualifying primes");
        return CBS_ERR_INVALID_ARG;
    }
    for (uint32_t i = 0; i < count; ++i) h_out[i] = v[i];
    return CBS_OK;
}

}  // extern "C"
