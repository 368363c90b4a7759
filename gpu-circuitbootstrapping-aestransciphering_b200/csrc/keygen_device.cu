// keygen_device.cu -- key generation on the device.
//
// The reference generates its keys in its OpenFHE fork on the host (KeyGen, RLWEKeyGen,
// CirBTKeyGen, KeySwitchGen at examples/aes_transcipher/main.cu:232-252) and re-lays them for
// the device in host loops with a synchronisation per key (gpu_init_cirbsk,
// bitwise/src/cirbts/cirbts-init.cu:367-864).  Here every word is drawn on the device from
// ChaCha20 under a 256-bit key, one block per coefficient, the block addressed by (counter,
// nonce = (sample, domain, 0)) so the words do not depend on the launch shape and the oracle
// restates each of them:
//   domain 3  secrets: s_lwe[i] = bit 0 of ChaCha20(i, (0, 3)); s_rlwe[i] = floor(3 x / 2^128) - 1
//             for x = words 0-3 of ChaCha20(i, (1, 3))
//   domain 4  BSK RGSW(s_i), sample i * 2 digits + row: RLWE(0), then g_j added to every NTT slot
//             of component a (row 2j) or b (row 2j + 1) when s_i = 1
//   domain 5  HomTrace keys, sample round * digits_ht + j: RLWE(0), b -= sigma_r(s) g_j
//   domain 6  SchemeSwitch key, sample j: RLWE(0), b += s^2 g_j
//   domain 7  extraction KSK, sample ((j N + i) base_ks + v): a[c] = floor(qks x / 2^128) from
//             ChaCha20(c, (t, 7)), noise from ChaCha20(n, (t, 7)) words 4-5, b = <a, s> +
//             v s'_i base_ks^j + e mod qks
//   domain 8 / 9 / 10  grouped keys for mb = 2 / 3 / 4, sample (group * keys + subset) * 2 digits
//             + row: RLWE(0), g_j added as for the BSK when prod_{i in subset} s_i = 1
// RLWE(0) samples are those of the AES-material encryption (encrypt.cu): NTT-domain mask from
// words 0-3, discrete-Gaussian noise from words 4-5, b = a s + NTT(e).
#include <sys/random.h>

#include <algorithm>
#include <cerrno>
#include <cstring>
#include <string>
#include <vector>

#include "chacha.cuh"
#include "common.cuh"
#include "context.cuh"
#include "encrypt.cuh"

namespace cbs {

__global__ void k_keygen_secrets(ChachaKey k, uint32_t n, uint32_t N, int32_t* s_lwe, int32_t* s_rlwe) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t blk[6];
    if (i < n) {
        chacha20_block(k, i, 0u, 3u, blk);
        s_lwe[i] = static_cast<int32_t>(blk[0] & 1u);
    }
    if (i < N) {
        chacha20_block(k, i, 1u, 3u, blk);
        s_rlwe[i] = static_cast<int32_t>(uniform_mod(blk, 3)) - 1;
    }
}

// RGSW messages of the bootstrapping keys: sample (u, row) of an RLWE(0) batch [count][l2][2][N]
// gets g_(row/2) on every NTT slot of component row % 2 when bit[u] is set
__global__ void k_keygen_rgsw_message(uint64_t* keys, const uint8_t* bit, const uint64_t* g, uint32_t count,
                                      uint32_t l2, uint32_t N, uint64_t Q) {
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t total = static_cast<size_t>(count) * l2 * N;
    if (idx >= total) return;
    const uint32_t c = static_cast<uint32_t>(idx % N);
    const size_t rowi = idx / N;
    const uint32_t row = static_cast<uint32_t>(rowi % l2), u = static_cast<uint32_t>(rowi / l2);
    if (!bit[u]) return;
    uint64_t* p = keys + (rowi * 2 + (row & 1u)) * N + c;
    *p = add_mod(*p, g[row >> 1], Q);
}

// key-switching messages: b[s] += sign * msg[s / digits] * g[s % digits] (NTT domain)
__global__ void k_keygen_switch_message(uint64_t* keys, const uint64_t* msg, const uint64_t* g, uint32_t count,
                                        uint32_t digits, uint32_t N, uint64_t Q, uint64_t r0, uint64_t r1, int sub) {
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<size_t>(count) * N) return;
    const uint32_t c = static_cast<uint32_t>(idx % N), smp = static_cast<uint32_t>(idx / N);
    const uint64_t m = mul_mod_barrett(msg[static_cast<size_t>(smp / digits) * N + c], g[smp % digits], Q, r0, r1);
    uint64_t* b = keys + (static_cast<size_t>(smp) * 2 + 1) * N + c;
    *b = sub ? sub_mod(*b, m, Q) : add_mod(*b, m, Q);
}

// sigma_r(s) = s(X^(N/2^r + 1)) in the coefficient domain mod Q, [rounds][N]
__global__ void k_keygen_auto_secret(const int32_t* s_rlwe, uint32_t N, uint32_t rounds, uint64_t Q, uint64_t* sig) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
    if (i >= N || r >= rounds) return;
    const uint64_t kk = (static_cast<uint64_t>(N) >> r) + 1;
    const uint64_t e = (static_cast<uint64_t>(i) * kk) % (2ull * N);
    const int32_t v = e < N ? s_rlwe[i] : -s_rlwe[i];
    sig[static_cast<size_t>(r) * N + (e % N)] = v < 0 ? Q - static_cast<uint64_t>(-v) : static_cast<uint64_t>(v);
}

// s mod Q (coefficient domain) and s^2 (NTT domain, from NTT(s))
__global__ void k_keygen_secret_mod(const int32_t* s_rlwe, uint32_t N, uint64_t Q, uint64_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = s_rlwe[i] < 0 ? Q - 1 : static_cast<uint64_t>(s_rlwe[i]);
}
__global__ void k_keygen_square(const uint64_t* s_ntt, uint64_t* out, uint32_t N, uint64_t Q, uint64_t r0,
                                uint64_t r1) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = mul_mod_barrett(s_ntt[i], s_ntt[i], Q, r0, r1);
}

// extraction key switch N -> n, one CTA per LWE sample, block-reduced <a, s> (u16 words, qks <= 2^16)
// rows written row_stride words apart (the extraction kernel's padded layout, pad words zero)
__global__ void k_keygen_ksk(ChachaKey k, const int32_t* s_lwe, const int32_t* s_rlwe, uint16_t* ksk, uint32_t n,
                             uint32_t N, uint32_t base, uint32_t qks, const uint64_t* cdt, uint32_t cdt_len,
                             uint32_t row_stride) {
    __shared__ uint32_t part[32];
    const uint32_t t = blockIdx.x;
    const uint32_t v = t % base, i = (t / base) % N, j = t / (base * N);
    uint16_t* row = ksk + static_cast<size_t>(t) * row_stride;
    for (uint32_t c = n + 1 + threadIdx.x; c < row_stride; c += blockDim.x) row[c] = 0;
    uint32_t acc = 0;
    for (uint32_t c = threadIdx.x; c < n; c += blockDim.x) {
        uint32_t blk[6];
        chacha20_block(k, c, t, 7u, blk);
        const uint32_t a = static_cast<uint32_t>(uniform_mod(blk, qks));
        row[c] = static_cast<uint16_t>(a);
        acc += s_lwe[c] ? a : 0u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t sum = 0;
        for (uint32_t w = 0; w < (blockDim.x + 31) / 32; ++w) sum += part[w];
        uint32_t blk[6];
        chacha20_block(k, n, t, 7u, blk);
        const int64_t e = cdt_sample(blk, cdt, cdt_len);
        const uint32_t mask = qks - 1;
        const uint32_t si = static_cast<uint32_t>(s_rlwe[i] + static_cast<int32_t>(qks)) & mask;
        const uint32_t bj = j == 0 ? 1u : base;
        const uint32_t m = (v * si * bj) & mask;
        row[n] = static_cast<uint16_t>((sum + m + static_cast<uint32_t>(static_cast<int32_t>(e))) & mask);
    }
}

// NTT-domain key words to the Montgomery form the exact kernels read: x 2^64 mod Q
__global__ void k_keygen_to_mont(uint64_t* out, const uint64_t* in, size_t count, uint64_t r, uint64_t rs, uint64_t Q) {
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        out[i] = mul_shoup(in[i], r, rs, Q);
}

static cudaError_t to_mont_device(const cbs_context* c, DevBuf<uint64_t>& out, const uint64_t* in, size_t count,
                                  cudaStream_t s) {
    cudaError_t e = out.alloc(count);
    if (e != cudaSuccess) return e;
    const unsigned blocks = static_cast<unsigned>(std::min<size_t>((count + 255) / 256, 148u * 32u));
    k_keygen_to_mont<<<blocks ? blocks : 1, 256, 0, s>>>(out.p, in, count, c->mont_r, host::shoup(c->mont_r, c->p.Q),
                                                         c->p.Q);
    return cudaGetLastError();
}

static cudaError_t rlwe_zero_batch(const cbs_context* c, const ChachaKey& k, uint32_t domain, uint32_t count,
                                   uint64_t* out, uint64_t* tmp, const uint64_t* d_s_ntt, const DevBuf<uint64_t>& cdt,
                                   uint32_t cdt_len, cudaStream_t s) {
    EncryptRlweArgs ra{};
    ra.key = k;
    ra.words = nullptr;
    ra.ct = out;
    ra.tmp = tmp;
    ra.s_ntt = d_s_ntt;
    ra.cdt = cdt.p;
    ra.cdt_len = cdt_len;
    ra.N = c->p.N;
    ra.first = 0;
    ra.Q = c->p.Q;
    ra.delta = 0;
    ra.ratio0 = c->tab.ratio0;
    ra.ratio1 = c->tab.ratio1;
    ra.domain = domain;
    return launch_encrypt_rlwe_words(ra, count, c->d_rp.p, c->d_rps.p, c->d_mod.p, s);
}

static std::vector<uint64_t> gadget_powers(uint64_t Q, uint32_t base, uint32_t digits) {
    int gb = 0;
    while ((1u << gb) < base) ++gb;
    int logq = 0;
    while (logq < 64 && (Q >> logq)) ++logq;
    int ign = logq - static_cast<int>(digits) * gb;
    if (ign < 0) ign = 0;
    std::vector<uint64_t> g(digits);
    for (uint32_t j = 0; j < digits; ++j) g[j] = (1ull << (ign + static_cast<int>(j) * gb)) % Q;
    return g;
}

static bool os_random_key(ChachaKey& k) {
    uint8_t* out = reinterpret_cast<uint8_t*>(k.w);
    size_t got = 0;
    while (got < sizeof(k.w)) {
        const ssize_t r = getrandom(out + got, sizeof(k.w) - got, 0);
        if (r < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        got += static_cast<size_t>(r);
    }
    return true;
}

// the grouped keys of the device-generated key set (domain 8 / 9 / 10) into c->h_mbk
cbs_status device_grouped_keys(cbs_context* c, uint32_t mb) {
    const uint32_t N = c->p.N, n = c->p.n, l2 = 2 * c->p.digits_g, K = mb_subsets(mb), groups = (n + mb - 1) / mb;
    cudaStream_t s = c->stream;
    const auto cdt_r = cdt_table(c->p.sigma_rlwe);
    DevBuf<uint64_t> d_cdt, d_s_ntt, d_g, d_keys, d_tmp;
    DevBuf<uint8_t> d_bit;
    if (!cdt_r.empty()) CBS_CUDA_TRY(d_cdt.upload(cdt_r.data(), cdt_r.size(), s));
    CBS_CUDA_TRY(d_s_ntt.upload(c->hk.s_ntt.data(), N, s));
    const auto g = gadget_powers(c->p.Q, c->p.base_g, c->p.digits_g);
    CBS_CUDA_TRY(d_g.upload(g.data(), g.size(), s));
    std::vector<uint8_t> bits(static_cast<size_t>(groups) * K);
    for (uint32_t gi = 0; gi < groups; ++gi)
        for (uint32_t kk = 0; kk < K; ++kk) {
            const uint32_t mask = mb_subset_mask(mb, kk);
            uint32_t prod = 1;
            for (uint32_t i = 0; i < mb; ++i)
                if (mask & (1u << i)) {
                    const uint32_t idx = gi * mb + i;
                    prod &= idx < n ? static_cast<uint32_t>(c->hk.s_lwe[idx]) : 0u;
                }
            bits[static_cast<size_t>(gi) * K + kk] = static_cast<uint8_t>(prod);
        }
    CBS_CUDA_TRY(d_bit.upload(bits.data(), bits.size(), s));
    const size_t samples = bits.size() * l2;
    CBS_CUDA_TRY(d_keys.alloc(samples * 2 * N));
    CBS_CUDA_TRY(d_tmp.alloc(samples * N));
    CBS_CUDA_TRY(rlwe_zero_batch(c, c->keygen_key, mb == 2 ? 8u : (mb == 3 ? 9u : 10u), static_cast<uint32_t>(samples), d_keys.p,
                                 d_tmp.p, d_s_ntt.p, d_cdt, static_cast<uint32_t>(cdt_r.size()), s));
    const size_t work = samples * N;
    k_keygen_rgsw_message<<<static_cast<unsigned>((work + 255) / 256), 256, 0, s>>>(
        d_keys.p, d_bit.p, d_g.p, static_cast<uint32_t>(bits.size()), l2, N, c->p.Q);
    CBS_CUDA_TRY(cudaGetLastError());
    c->h_mbk.resize(samples * 2 * N);
    CBS_CUDA_TRY(cudaMemcpyAsync(c->h_mbk.data(), d_keys.p, c->h_mbk.size() * 8, cudaMemcpyDeviceToHost, s));
    CBS_CUDA_TRY(cudaStreamSynchronize(s));
    return CBS_OK;
}

}  // namespace cbs

using namespace cbs;

extern "C" {

cbs_status cbs_keygen_device(cbs_context* ctx, const uint8_t* rng_key) {
    CBS_CHECK_ARG(ctx, "keygen_device: null context");
    cbs_context* c = ctx;
    ChachaKey k{};
    if (rng_key) {
        std::memcpy(k.w, rng_key, 32);
    } else if (!os_random_key(k)) {
        set_error(std::string("keygen_device: getrandom failed: ") + std::strerror(errno));
        return CBS_ERR_UNSUPPORTED;
    }
    const cbs_params& p = c->p;
    const uint32_t N = p.N, n = p.n, l2 = 2 * p.digits_g, rounds = c->rounds;
    const uint64_t Q = p.Q;
    cudaStream_t s = c->stream;
    c->keys_ready = false;  // until the new keys are in place
    c->aes.ready = false;
    c->aes.drop_graphs();

    // secrets
    DevBuf<int32_t> d_s_lwe, d_s_rlwe;
    CBS_CUDA_TRY(d_s_lwe.alloc(n));
    CBS_CUDA_TRY(d_s_rlwe.alloc(N));
    const uint32_t span = n > N ? n : N;
    k_keygen_secrets<<<(span + 255) / 256, 256, 0, s>>>(k, n, N, d_s_lwe.p, d_s_rlwe.p);
    CBS_CUDA_TRY(cudaGetLastError());
    HostKeys& hk = c->hk;
    hk = HostKeys{};
    hk.s_lwe.resize(n);
    hk.s_rlwe.resize(N);
    CBS_CUDA_TRY(cudaMemcpyAsync(hk.s_lwe.data(), d_s_lwe.p, n * 4ull, cudaMemcpyDeviceToHost, s));
    CBS_CUDA_TRY(cudaMemcpyAsync(hk.s_rlwe.data(), d_s_rlwe.p, N * 4ull, cudaMemcpyDeviceToHost, s));
    DevBuf<uint64_t> d_s_ntt, d_s2, d_sig, d_g, d_cdt_r, d_cdt_l, d_keys, d_tmp;
    CBS_CUDA_TRY(d_s_ntt.alloc(N));
    k_keygen_secret_mod<<<(N + 255) / 256, 256, 0, s>>>(d_s_rlwe.p, N, Q, d_s_ntt.p);
    CBS_CUDA_TRY(cudaGetLastError());
    CBS_CUDA_TRY(ntt_forward(d_s_ntt.p, d_s_ntt.p, c->d_rp.p, c->d_rps.p, c->d_mod.p, N, 1, s));
    hk.s_ntt.resize(N);
    CBS_CUDA_TRY(cudaMemcpyAsync(hk.s_ntt.data(), d_s_ntt.p, N * 8ull, cudaMemcpyDeviceToHost, s));
    const auto cdt_r = cdt_table(p.sigma_rlwe), cdt_l = cdt_table(p.sigma_lwe);
    if (!cdt_r.empty()) CBS_CUDA_TRY(d_cdt_r.upload(cdt_r.data(), cdt_r.size(), s));
    if (!cdt_l.empty()) CBS_CUDA_TRY(d_cdt_l.upload(cdt_l.data(), cdt_l.size(), s));
    const uint32_t lr = static_cast<uint32_t>(cdt_r.size()), ll = static_cast<uint32_t>(cdt_l.size());

    // bootstrapping key
    const size_t bsk_samples = static_cast<size_t>(n) * l2;
    const size_t big = std::max({bsk_samples, static_cast<size_t>(rounds) * p.digits_ht, static_cast<size_t>(p.digits_ss)});
    CBS_CUDA_TRY(d_keys.alloc(big * 2 * N));
    CBS_CUDA_TRY(d_tmp.alloc(big * N));
    const auto gbr = gadget_powers(Q, p.base_g, p.digits_g);
    CBS_CUDA_TRY(d_g.upload(gbr.data(), gbr.size(), s));
    CBS_CUDA_TRY(rlwe_zero_batch(c, k, 4u, static_cast<uint32_t>(bsk_samples), d_keys.p, d_tmp.p, d_s_ntt.p, d_cdt_r,
                                 lr, s));
    {
        DevBuf<uint8_t> d_bit;
        std::vector<uint8_t> bit(n);
        CBS_CUDA_TRY(cudaStreamSynchronize(s));  // the secrets are on the host now
        for (uint32_t i = 0; i < n; ++i) bit[i] = static_cast<uint8_t>(hk.s_lwe[i]);
        CBS_CUDA_TRY(d_bit.upload(bit.data(), n, s));
        const size_t work = bsk_samples * N;
        k_keygen_rgsw_message<<<static_cast<unsigned>((work + 255) / 256), 256, 0, s>>>(d_keys.p, d_bit.p, d_g.p, n, l2,
                                                                                          N, Q);
        CBS_CUDA_TRY(cudaGetLastError());
        hk.bsk.resize(bsk_samples * 2 * N);
        CBS_CUDA_TRY(cudaMemcpyAsync(hk.bsk.data(), d_keys.p, hk.bsk.size() * 8, cudaMemcpyDeviceToHost, s));
        CBS_CUDA_TRY(to_mont_device(c, c->d_bsk, d_keys.p, hk.bsk.size(), s));
        CBS_CUDA_TRY(cudaStreamSynchronize(s));
    }

    // HomTrace keys: b -= sigma_r(s) g_j
    {
        const uint32_t cnt = rounds * p.digits_ht;
        CBS_CUDA_TRY(d_sig.alloc(static_cast<size_t>(rounds) * N));
        k_keygen_auto_secret<<<dim3((N + 255) / 256, rounds), 256, 0, s>>>(d_s_rlwe.p, N, rounds, Q, d_sig.p);
        CBS_CUDA_TRY(cudaGetLastError());
        CBS_CUDA_TRY(ntt_forward(d_sig.p, d_sig.p, c->d_rp.p, c->d_rps.p, c->d_mod.p, N, rounds, s));
        const auto ght = gadget_powers(Q, p.base_ht, p.digits_ht);
        CBS_CUDA_TRY(d_g.upload(ght.data(), ght.size(), s));
        CBS_CUDA_TRY(rlwe_zero_batch(c, k, 5u, cnt, d_keys.p, d_tmp.p, d_s_ntt.p, d_cdt_r, lr, s));
        const size_t work = static_cast<size_t>(cnt) * N;
        k_keygen_switch_message<<<static_cast<unsigned>((work + 255) / 256), 256, 0, s>>>(
            d_keys.p, d_sig.p, d_g.p, cnt, p.digits_ht, N, Q, c->tab.ratio0, c->tab.ratio1, 1);
        CBS_CUDA_TRY(cudaGetLastError());
        hk.ht.resize(static_cast<size_t>(cnt) * 2 * N);
        CBS_CUDA_TRY(cudaMemcpyAsync(hk.ht.data(), d_keys.p, hk.ht.size() * 8, cudaMemcpyDeviceToHost, s));
        CBS_CUDA_TRY(to_mont_device(c, c->d_ht, d_keys.p, hk.ht.size(), s));
        CBS_CUDA_TRY(cudaStreamSynchronize(s));
    }

    // SchemeSwitch key: b += s^2 g_j
    {
        const uint32_t cnt = p.digits_ss;
        CBS_CUDA_TRY(d_s2.alloc(N));
        k_keygen_square<<<(N + 255) / 256, 256, 0, s>>>(d_s_ntt.p, d_s2.p, N, Q, c->tab.ratio0, c->tab.ratio1);
        CBS_CUDA_TRY(cudaGetLastError());
        const auto gss = gadget_powers(Q, p.base_ss, p.digits_ss);
        CBS_CUDA_TRY(d_g.upload(gss.data(), gss.size(), s));
        CBS_CUDA_TRY(rlwe_zero_batch(c, k, 6u, cnt, d_keys.p, d_tmp.p, d_s_ntt.p, d_cdt_r, lr, s));
        const size_t work = static_cast<size_t>(cnt) * N;
        k_keygen_switch_message<<<static_cast<unsigned>((work + 255) / 256), 256, 0, s>>>(
            d_keys.p, d_s2.p, d_g.p, cnt, cnt, N, Q, c->tab.ratio0, c->tab.ratio1, 0);
        CBS_CUDA_TRY(cudaGetLastError());
        hk.ss.resize(static_cast<size_t>(cnt) * 2 * N);
        CBS_CUDA_TRY(cudaMemcpyAsync(hk.ss.data(), d_keys.p, hk.ss.size() * 8, cudaMemcpyDeviceToHost, s));
        CBS_CUDA_TRY(to_mont_device(c, c->d_ss, d_keys.p, hk.ss.size(), s));
        CBS_CUDA_TRY(cudaStreamSynchronize(s));
    }

    // extraction key switch
    {
        const size_t samples = static_cast<size_t>(2) * N * p.base_ks;
        // written straight into the context's padded device key; exported on demand
        const uint32_t stride = ksk_row_stride(n);
        CBS_CUDA_TRY(c->d_ksk.alloc(samples * stride));
        k_keygen_ksk<<<static_cast<unsigned>(samples), 128, 0, s>>>(k, d_s_lwe.p, d_s_rlwe.p, c->d_ksk.p, n, N,
                                                                     p.base_ks, p.qks, d_cdt_l.p, ll, stride);
        CBS_CUDA_TRY(cudaGetLastError());
        CBS_CUDA_TRY(cudaStreamSynchronize(s));
        c->ksk_device_only = true;
    }
    derive_key_tables(p, hk);
    c->keygen_key = k;
    c->device_keyed = true;
    c->has_secret = true;
    c->key_seed = 0;
    volatile uint32_t* wipe = k.w;
    for (int i = 0; i < 8; ++i) wipe[i] = 0;
    return finish_key_upload(c);
}

}  // extern "C"
