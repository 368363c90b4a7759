// ntt.cu -- batched single-modulus negacyclic NTT/INTT (Phantom 1-D API) on sm_100a.
//
// Drop-in for src/ntt/ntt_1d.cu:760-789 (fnwt_1d_opt_batched, inwt_1d_opt_batched,
// inwt_1d_opt_outofplace_batched, inwt_1d_opt_permute_batched): same tables, same
// argument meaning, bit-identical outputs.  One polynomial per CTA, N/8 threads, the
// register-blocked transform of ntt_core.cuh.
#include "common.cuh"
#include "ntt_core.cuh"

namespace cbs {

template <int LOGN>
__global__ void __launch_bounds__(NttPlan<LOGN>::T) k_fnwt(uint64_t* __restrict__ out, const uint64_t* __restrict__ in,
                                                           const uint64_t* __restrict__ tw,
                                                           const uint64_t* __restrict__ tws,
                                                           const cbs_dmodulus* __restrict__ mod, size_t batch) {
    __shared__ uint64_t sm[1 << LOGN];
    const size_t poly = blockIdx.x;
    if (poly >= batch) return;
    const uint64_t q = mod->value;
    const uint64_t* src = in + (poly << LOGN);
    uint64_t* dst = out + (poly << LOGN);
    ntt_forward_cta<LOGN>(
        sm, threadIdx.x, tw, tws, q, [&](uint32_t i) { return src[i]; },
        [&](int, uint32_t i, uint64_t v) { dst[i] = v; });
}

template <int LOGN>
__global__ void __launch_bounds__(NttPlan<LOGN>::T) k_inwt(uint64_t* __restrict__ out, const uint64_t* __restrict__ in,
                                                           const uint32_t* __restrict__ map,
                                                           const uint64_t* __restrict__ itw,
                                                           const uint64_t* __restrict__ itws,
                                                           const cbs_dmodulus* __restrict__ mod,
                                                           const uint64_t* __restrict__ scalar,
                                                           const uint64_t* __restrict__ scalar_shoup, size_t batch) {
    __shared__ uint64_t sm[1 << LOGN];
    constexpr uint32_t N = 1u << LOGN;
    const size_t poly = blockIdx.x;
    if (poly >= batch) return;
    const uint64_t q = mod->value;
    const uint64_t ninv = *scalar, ninv_s = *scalar_shoup;
    const uint64_t* src = in + (poly << LOGN);
    uint64_t* dst = out + (poly << LOGN);
    if (map == nullptr) {
        ntt_inverse_cta<LOGN>(
            sm, threadIdx.x, itw, itws, ninv, ninv_s, q, [&](int, uint32_t i) { return src[i]; },
            [&](uint32_t i, uint64_t v) { dst[i] = v; });
    } else {
        // permute variant (ntt_1d.cu:677-757): slot i reads in[map[i]], negated when map[i] >= N
        ntt_inverse_cta<LOGN>(
            sm, threadIdx.x, itw, itws, ninv, ninv_s, q,
            [&](int, uint32_t i) {
                uint32_t s = __ldg(map + i);
                const bool neg = s >= N;
                s -= neg ? N : 0u;
                const uint64_t v = src[s];
                return (neg && v) ? q - v : v;
            },
            [&](uint32_t i, uint64_t v) { dst[i] = v; });
    }
}

template <int LOGN>
static cudaError_t launch_fwd(uint64_t* out, const uint64_t* in, const uint64_t* tw, const uint64_t* tws,
                              const cbs_dmodulus* mod, size_t batch, cudaStream_t s) {
    k_fnwt<LOGN><<<static_cast<unsigned>(batch), NttPlan<LOGN>::T, 0, s>>>(out, in, tw, tws, mod, batch);
    return cudaGetLastError();
}

template <int LOGN>
static cudaError_t launch_inv(uint64_t* out, const uint64_t* in, const uint32_t* map, const uint64_t* itw,
                              const uint64_t* itws, const cbs_dmodulus* mod, const uint64_t* sc, const uint64_t* scs,
                              size_t batch, cudaStream_t s) {
    k_inwt<LOGN><<<static_cast<unsigned>(batch), NttPlan<LOGN>::T, 0, s>>>(out, in, map, itw, itws, mod, sc, scs,
                                                                           batch);
    return cudaGetLastError();
}

cudaError_t ntt_forward(uint64_t* out, const uint64_t* in, const uint64_t* tw, const uint64_t* tws,
                        const cbs_dmodulus* mod, size_t dim, size_t batch, cudaStream_t s) {
    if (batch == 0) return cudaSuccess;
    switch (ilog2(dim)) {
        case 10: return launch_fwd<10>(out, in, tw, tws, mod, batch, s);
        case 11: return launch_fwd<11>(out, in, tw, tws, mod, batch, s);
        case 12: return launch_fwd<12>(out, in, tw, tws, mod, batch, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t ntt_inverse(uint64_t* out, const uint64_t* in, const uint32_t* map, const uint64_t* itw,
                        const uint64_t* itws, const cbs_dmodulus* mod, const uint64_t* sc, const uint64_t* scs,
                        size_t dim, size_t batch, cudaStream_t s) {
    if (batch == 0) return cudaSuccess;
    switch (ilog2(dim)) {
        case 10: return launch_inv<10>(out, in, map, itw, itws, mod, sc, scs, batch, s);
        case 11: return launch_inv<11>(out, in, map, itw, itws, mod, sc, scs, batch, s);
        case 12: return launch_inv<12>(out, in, map, itw, itws, mod, sc, scs, batch, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace cbs
