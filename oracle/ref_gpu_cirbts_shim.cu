// ref_gpu_cirbts_shim.cu -- drives the reference's own one-bit GINX blind-rotation kernels,
// compiled for sm_100a from bitwise/src/cirbts/kernel.cu and src/ntt/ntt_1d.cu where they lie
// (`make -C oracle ref_gpu_cirbts`, stand-in headers in ref_shim_cirbts/), in the launch
// sequence of the reference's batched blind rotation (bitwise/src/cirbts/cirbts-batch.cu:
// 3438-3446 index positions, 4064-4075 per-step INTT + fused decomposition/NTT, 3976-3980
// binary MAC with the AoS key).  Test infrastructure only: the GPU tests compare the
// accumulator it produces with the oracle's, which the product's NTT path matches bit for bit.
#include <cstdint>
#include <utility>
#include <vector>

#include "cirbts/kernel.cuh"
#include "ntt.cuh"

extern "C" {

// Shoup quotients floor(w 2^64 / Q) of count words (host), as the reference's key tables
void ref_cirbts_shoup(const uint64_t* w, uint64_t* out, size_t count, uint64_t Q) {
    for (size_t i = 0; i < count; ++i)
        out[i] = static_cast<uint64_t>((static_cast<unsigned __int128>(w[i]) << 64) / Q);
}

// n steps of the one-bit blind rotation on acc [batch][2][N] (NTT domain, updated in place):
// ek / ek_shoup [n][2 digits][2][N] (the reference's AoS RF key and its Shoup table), monic
// [2N][N] = NTT(X^k - 1) (cirbts-init.cu:991-1010), d_a [batch][a_stride] LWE masks mod q_lwe,
// Phantom tables and DModulus as the product's cbs_ntt_tables_host builds them.  Returns the
// CUDA error code (0 on success).
int ref_cirbts_blind_rotate_steps(uint64_t* acc, const uint64_t* d_a, uint32_t a_stride, uint32_t n, uint32_t batch,
                                  const uint64_t* ek, const uint64_t* ek_shoup, const uint64_t* monic,
                                  const void* d_mod, const uint64_t* tw, const uint64_t* tws, const uint64_t* itw,
                                  const uint64_t* itws, const uint64_t* ninv, const uint64_t* ninv_s, uint32_t N,
                                  uint64_t Q, uint32_t base_g, uint32_t digits_g, uint64_t q_lwe, uint32_t bitwidth,
                                  void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const DModulus* mod = static_cast<const DModulus*>(d_mod);
    const uint32_t digitsG2 = 2 * digits_g, twoN = 2 * N;
    uint64_t *ct = nullptr, *dct = nullptr;
    uint32_t* index_pos = nullptr;
    cudaError_t e = cudaMalloc(&ct, sizeof(uint64_t) * 2 * N * batch);
    if (e == cudaSuccess) e = cudaMalloc(&dct, sizeof(uint64_t) * digitsG2 * N * batch);
    if (e == cudaSuccess) e = cudaMalloc(&index_pos, sizeof(uint32_t) * n * batch);
    if (e == cudaSuccess) {
        const dim3 ms_block(256), ms_grid((n + 255) / 256, batch);
        kernel_SpecialMS_IndexPos_Batch<<<ms_grid, ms_block, 0, s>>>(d_a, index_pos, n, batch, a_stride, twoN, q_lwe,
                                                                     bitwidth);
        const uint32_t tpb = N / 2 < 256 ? N / 2 : 256;
        const dim3 eb(256), eg((N + 255) / 256, batch);
        for (uint32_t i = 0; i < n && e == cudaSuccess; ++i) {
            inwt_1d_opt_outofplace_batched(ct, acc, itw, itws, mod, ninv, ninv_s, N, static_cast<size_t>(2) * batch,
                                           s);
            kernel_SignedDigitDecompose2_FusedFNWT_Batch<<<digitsG2 * batch, tpb, N * sizeof(uint64_t), s>>>(
                dct, ct, Q, base_g, digits_g, N, batch, tw, tws, mod);
            kernel_EvalAccCore_Binary_Batch<<<eg, eb, 0, s>>>(acc, dct, ek, ek_shoup, monic, N, mod, digitsG2, i,
                                                              index_pos, n);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaFree(ct);
    cudaFree(dct);
    cudaFree(index_pos);
    return static_cast<int>(e);
}

// Grouped (mb = 2) blind rotation in the reference's CIRBTS_PBS_MULTIBIT=2 launch sequence
// (bitwise/src/cirbts/cirbts-batch.cu:4402-4470): per group the INTT and fused
// decomposition/NTT, then kernel_EvalAccCore_Binary_MB2_Grouped_Batch (or the one-key grouped
// kernel for an odd tail coefficient).  ek / ek_shoup: the reference's grouped RF key
// [3 subsets {0} {1} {0,1}][ceil(n/2)][2 digits][2][N] and its Shoup table; the rest as
// ref_cirbts_blind_rotate_steps.
int ref_cirbts_blind_rotate_mb2(uint64_t* acc, const uint64_t* d_a, uint32_t a_stride, uint32_t n, uint32_t batch,
                                const uint64_t* ek, const uint64_t* ek_shoup, const uint64_t* monic, const void* d_mod,
                                const uint64_t* tw, const uint64_t* tws, const uint64_t* itw, const uint64_t* itws,
                                const uint64_t* ninv, const uint64_t* ninv_s, uint32_t N, uint64_t Q, uint32_t base_g,
                                uint32_t digits_g, uint64_t q_lwe, uint32_t bitwidth, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const DModulus* mod = static_cast<const DModulus*>(d_mod);
    const uint32_t digitsG2 = 2 * digits_g, twoN = 2 * N, groups = (n + 1) / 2;
    const size_t key_block = static_cast<size_t>(groups) * digitsG2 * 2 * N;
    uint64_t *ct = nullptr, *dct = nullptr;
    uint32_t* index_pos = nullptr;
    cudaError_t e = cudaMalloc(&ct, sizeof(uint64_t) * 2 * N * batch);
    if (e == cudaSuccess) e = cudaMalloc(&dct, sizeof(uint64_t) * digitsG2 * N * batch);
    if (e == cudaSuccess) e = cudaMalloc(&index_pos, sizeof(uint32_t) * n * batch);
    if (e == cudaSuccess) {
        kernel_SpecialMS_IndexPos_Batch<<<dim3((n + 255) / 256, batch), 256, 0, s>>>(d_a, index_pos, n, batch, a_stride,
                                                                                     twoN, q_lwe, bitwidth);
        const uint32_t tpb = N / 2 < 256 ? N / 2 : 256;
        const dim3 eb(256), eg((N + 255) / 256, batch);
        for (uint32_t g = 0; g < groups && e == cudaSuccess; ++g) {
            const uint32_t idx0 = 2 * g, idx1 = idx0 + 1;
            inwt_1d_opt_outofplace_batched(ct, acc, itw, itws, mod, ninv, ninv_s, N, static_cast<size_t>(2) * batch,
                                           s);
            kernel_SignedDigitDecompose2_FusedFNWT_Batch<<<digitsG2 * batch, tpb, N * sizeof(uint64_t), s>>>(
                dct, ct, Q, base_g, digits_g, N, batch, tw, tws, mod);
            if (idx1 < n)
                kernel_EvalAccCore_Binary_MB2_Grouped_Batch<<<eg, eb, 0, s>>>(
                    acc, dct, ek, ek_shoup, ek + key_block, ek_shoup + key_block, ek + 2 * key_block,
                    ek_shoup + 2 * key_block, monic, N, mod, digitsG2, g, idx0, idx1, index_pos, n);
            else
                kernel_EvalAccCore_Binary_Grouped_Batch<<<eg, eb, 0, s>>>(acc, dct, ek, ek_shoup, monic, N, mod, digitsG2,
                                                                          g, idx0, index_pos, n);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaFree(ct);
    cudaFree(dct);
    cudaFree(index_pos);
    return static_cast<int>(e);
}

// Staged grouped (mb = 4, CIRBTS_PBS_MULTIBIT=4) blind rotation in the reference's launch
// sequence (bitwise/src/cirbts/cirbts-batch.cu:2767-2923, AoS keys): per group of 4, the INTT
// and fused decomposition/NTT, then kernel_EvalAccCore_Binary_MB3_Grouped_Batch on coefficients
// 0-2 (the MB2 grouped or one-key kernel for a shorter tail); then, when the group has a fourth
// coefficient, a fresh INTT and decomposition/NTT and the one-key kernel with key 3.
// ek / ek_shoup: the reference's 8-slot grouped RF key [8 {0} {1} {2} {3} {0,1} {0,2} {1,2}
// {0,1,2}][ceil(n/4)][2 digits][2][N] (cirbts-init.cu:536-565) and its Shoup table; the rest as
// ref_cirbts_blind_rotate_steps.
int ref_cirbts_blind_rotate_mb4(uint64_t* acc, const uint64_t* d_a, uint32_t a_stride, uint32_t n, uint32_t batch,
                                const uint64_t* ek, const uint64_t* ek_shoup, const uint64_t* monic, const void* d_mod,
                                const uint64_t* tw, const uint64_t* tws, const uint64_t* itw, const uint64_t* itws,
                                const uint64_t* ninv, const uint64_t* ninv_s, uint32_t N, uint64_t Q, uint32_t base_g,
                                uint32_t digits_g, uint64_t q_lwe, uint32_t bitwidth, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const DModulus* mod = static_cast<const DModulus*>(d_mod);
    const uint32_t digitsG2 = 2 * digits_g, twoN = 2 * N, groups = (n + 3) / 4;
    const size_t key_block = static_cast<size_t>(groups) * digitsG2 * 2 * N;
    const uint64_t* k[8];
    const uint64_t* ks[8];
    for (int i = 0; i < 8; ++i) {
        k[i] = ek + i * key_block;
        ks[i] = ek_shoup + i * key_block;
    }
    uint64_t *ct = nullptr, *dct = nullptr;
    uint32_t* index_pos = nullptr;
    cudaError_t e = cudaMalloc(&ct, sizeof(uint64_t) * 2 * N * batch);
    if (e == cudaSuccess) e = cudaMalloc(&dct, sizeof(uint64_t) * digitsG2 * N * batch);
    if (e == cudaSuccess) e = cudaMalloc(&index_pos, sizeof(uint32_t) * n * batch);
    if (e == cudaSuccess) {
        kernel_SpecialMS_IndexPos_Batch<<<dim3((n + 255) / 256, batch), 256, 0, s>>>(d_a, index_pos, n, batch, a_stride,
                                                                                     twoN, q_lwe, bitwidth);
        const uint32_t tpb = N / 2 < 256 ? N / 2 : 256;
        const dim3 eb(128), eg((N + 127) / 128, batch);
        auto decompose = [&]() {
            inwt_1d_opt_outofplace_batched(ct, acc, itw, itws, mod, ninv, ninv_s, N, static_cast<size_t>(2) * batch,
                                           s);
            kernel_SignedDigitDecompose2_FusedFNWT_Batch<<<digitsG2 * batch, tpb, N * sizeof(uint64_t), s>>>(
                dct, ct, Q, base_g, digits_g, N, batch, tw, tws, mod);
        };
        for (uint32_t g = 0; g < groups && e == cudaSuccess; ++g) {
            const uint32_t idx0 = 4 * g, idx1 = idx0 + 1, idx2 = idx0 + 2, idx3 = idx0 + 3;
            decompose();
            if (idx2 < n)
                kernel_EvalAccCore_Binary_MB3_Grouped_Batch<<<eg, eb, 0, s>>>(
                    acc, dct, k[0], ks[0], k[1], ks[1], k[2], ks[2], k[4], ks[4], k[5], ks[5], k[6], ks[6], k[7], ks[7],
                    monic, N, mod, digitsG2, g, idx0, idx1, idx2, index_pos, n);
            else if (idx1 < n)
                kernel_EvalAccCore_Binary_MB2_Grouped_Batch<<<eg, eb, 0, s>>>(acc, dct, k[0], ks[0], k[1], ks[1], k[4],
                                                                              ks[4], monic, N, mod, digitsG2, g, idx0,
                                                                              idx1, index_pos, n);
            else
                kernel_EvalAccCore_Binary_Grouped_Batch<<<eg, eb, 0, s>>>(acc, dct, k[0], ks[0], monic, N, mod,
                                                                          digitsG2, g, idx0, index_pos, n);
            if (idx3 < n) {
                decompose();
                kernel_EvalAccCore_Binary_Grouped_Batch<<<eg, eb, 0, s>>>(acc, dct, k[3], ks[3], monic, N, mod,
                                                                          digitsG2, g, idx3, index_pos, n);
            }
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaFree(ct);
    cudaFree(dct);
    cudaFree(index_pos);
    return static_cast<int>(e);
}

// LMKCDEY_EvalAcc (bitwise/src/cirbts/cirbts-lmkcdey.cu:105-407; window > 1 is its
// CIRBTS_LMK_AUTOKEYS_WINDOW key set, :49-103, and apply_skip, :302-325) of one ciphertext
// in the reference's launch sequence, over the reference's own kernels: the bucket CSR built
// on the host from the signed base-5 logarithms of (-a) | 1, kernel_Permute_Only for the
// automorphisms, inwt/fnwt_1d_opt_batched, kernel_SignedDigitDecomposeLMKCDEY_Ciphertext /
// _Poly (first digit dropped), kernel_MultAdd and kernel_AddInPlace.  acc [2][N] device, NTT
// domain, updated in place; h_a [n] host, the masks mod 2N as EvalAcc receives them; eval
// [n][2 digits][2][N], autok [1 + num_auto_keys][digits][2][N] (NTT domain), maps
// [1 + num_auto_keys][N] device; digits is the reference's digitsG - 1.  Scratch is
// allocated once per call; returns the CUDA error code.
int ref_cirbts_lmkcdey_eval_acc(uint64_t* acc, const uint32_t* h_a, uint32_t n, const uint64_t* eval,
                                const uint64_t* autok, const uint32_t* maps, uint32_t num_auto_keys, uint32_t window,
                                const void* d_mod,
                                const uint64_t* tw, const uint64_t* tws, const uint64_t* itw, const uint64_t* itws,
                                const uint64_t* ninv, const uint64_t* ninv_s, uint32_t N, uint64_t Q, uint32_t base_g,
                                uint32_t digits, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const DModulus* mod = static_cast<const DModulus*>(d_mod);
    const uint32_t Nh = N / 2, M = 2 * N, mask = M - 1, buckets = 2 * Nh, digits2 = 2 * digits;
    // signed base-5 logarithms of the odd residues (the reference's logGen)
    std::vector<int32_t> log_gen(M, 0);
    {
        uint64_t v = 1;
        for (uint32_t w = 0; w < Nh; ++w) {
            log_gen[v] = static_cast<int32_t>(w);
            log_gen[M - v] = w == 0 ? static_cast<int32_t>(M) : -static_cast<int32_t>(w);
            v = (v * 5) % M;
        }
    }
    std::vector<uint32_t> bucket_of(n), offsets(buckets + 1, 0), items(n);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t odd = ((0u - (h_a[i] & mask)) & mask) | 1u;
        const int32_t index = log_gen[odd];
        bucket_of[i] = index == static_cast<int32_t>(M) ? buckets - 1 : static_cast<uint32_t>(index + (int32_t)(Nh - 1));
        ++offsets[bucket_of[i] + 1];
    }
    for (uint32_t b = 0; b < buckets; ++b) offsets[b + 1] += offsets[b];
    {
        std::vector<uint32_t> cursor(offsets);
        for (uint32_t i = 0; i < n; ++i) items[cursor[bucket_of[i]]++] = i;
    }
    uint64_t *ct = nullptr, *dct = nullptr, *pc0 = nullptr, *pc1 = nullptr, *dcta = nullptr, *ks0 = nullptr,
             *ks1 = nullptr;
    cudaError_t e = cudaSuccess;
    for (auto bp : {std::make_pair(&ct, 2 * N), std::make_pair(&dct, digits2 * N), std::make_pair(&pc0, N),
                    std::make_pair(&pc1, N), std::make_pair(&dcta, digits * N), std::make_pair(&ks0, N),
                    std::make_pair(&ks1, N)})
        if (e == cudaSuccess) e = cudaMalloc(bp.first, sizeof(uint64_t) * bp.second);
    const dim3 block(256), grid((N + 255) / 256);
    const size_t eval_stride = static_cast<size_t>(digits2) * 2 * N, auto_stride = static_cast<size_t>(digits) * 2 * N;
    auto add_to_acc = [&](uint32_t j) {
        cudaMemcpyAsync(ct, acc, 2 * N * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
        inwt_1d_opt_batched(ct, itw, itws, mod, ninv, ninv_s, N, 2, s);
        kernel_SignedDigitDecomposeLMKCDEY_Ciphertext<<<grid, block, 0, s>>>(dct, ct, Q, base_g, digits2, N);
        fnwt_1d_opt_batched(dct, tw, tws, mod, N, digits2, s);
        kernel_MultAdd<<<grid, block, 0, s>>>(acc, acc + N, dct, eval + j * eval_stride, mod, digits2, N, 1);
    };
    auto automorphism = [&](uint32_t k) {
        const uint32_t* map = maps + static_cast<size_t>(k) * N;
        kernel_Permute_Only<<<grid, block, 0, s>>>(pc1, acc + N, map, N, 1, Q);
        kernel_Permute_Only<<<grid, block, 0, s>>>(pc0, acc, map, N, 1, Q);
        cudaMemcpyAsync(acc + N, pc1, N * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
        inwt_1d_opt_batched(pc0, itw, itws, mod, ninv, ninv_s, N, 1, s);
        kernel_SignedDigitDecomposeLMKCDEY_Poly<<<grid, block, 0, s>>>(dcta, pc0, Q, base_g, digits, N);
        fnwt_1d_opt_batched(dcta, tw, tws, mod, N, digits, s);
        kernel_MultAdd<<<grid, block, 0, s>>>(ks0, ks1, dcta, autok + k * auto_stride, mod, digits, N, 1);
        cudaMemcpyAsync(acc, ks0, N * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
        kernel_AddInPlace<<<grid, block, 0, s>>>(acc + N, ks1, mod, N);
    };
    // the key set's powers and their indices (build_lmk_auto_pows: 2N - 5, then 5^1 .. 5^numAutoKeys,
    // or 5^1 .. 5^window and every window-th power below 5^(N/2), repeats skipped)
    const bool use_window = window > 1;
    std::vector<uint64_t> pows{M - 5};
    auto pow5 = [M](uint32_t k) {
        uint64_t v = 1;
        for (uint32_t i = 0; i < k; ++i) v = (v * 5) % M;
        return v;
    };
    auto push = [&](uint32_t k) {
        const uint64_t v = pow5(k);
        for (uint64_t w : pows)
            if (w == v) return;
        pows.push_back(v);
    };
    if (use_window) {
        for (uint32_t k = 1; k <= window; ++k) push(k);
        for (uint32_t k = window; k <= Nh - 1; k += window) push(k);
    } else {
        for (uint32_t k = 1; k <= num_auto_keys; ++k) push(k);
    }
    auto key_index_for_step = [&](uint32_t step) {
        const uint64_t v = pow5(step);
        for (uint32_t i = 0; i < pows.size(); ++i)
            if (pows[i] == v) return i;
        return 0u;
    };
    auto apply_skip = [&](uint32_t skip) {
        if (skip == 0) return;
        if (!use_window) {
            automorphism(key_index_for_step(skip));
            return;
        }
        const uint32_t q = skip / window, r = skip % window;
        if (q) automorphism(key_index_for_step(q * window));
        if (r) automorphism(key_index_for_step(r));
    };
    if (e == cudaSuccess) {
        kernel_Permute_Only<<<grid, block, 0, s>>>(pc1, acc + N, maps, N, 1, Q);
        cudaMemcpyAsync(acc + N, pc1, N * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
        for (int half = 0; half < 2; ++half) {
            uint32_t skips = 0;
            for (uint32_t i = Nh - 1; i > 0; --i) {
                const uint32_t b = half == 0 ? (Nh - 1) - i : (Nh - 1) + i;
                if (offsets[b] != offsets[b + 1]) {
                    if (skips != 0) {
                        if (use_window) apply_skip(skips);
                        else automorphism(skips);
                        skips = 0;
                    }
                    for (uint32_t pos = offsets[b]; pos < offsets[b + 1]; ++pos) add_to_acc(items[pos]);
                }
                ++skips;
                if (use_window) {
                    if (i == 1) {
                        apply_skip(skips);
                        skips = 0;
                    }
                } else if (skips == num_auto_keys || i == 1) {
                    automorphism(skips);
                    skips = 0;
                }
            }
            const uint32_t sb = half == 0 ? buckets - 1 : Nh - 1;
            for (uint32_t pos = offsets[sb]; pos < offsets[sb + 1]; ++pos) add_to_acc(items[pos]);
            if (half == 0) automorphism(0);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    for (uint64_t* b : {ct, dct, pc0, pc1, dcta, ks0, ks1}) cudaFree(b);
    return static_cast<int>(e);
}

// N-major index positions [n][batch] of the LWE masks (kernel_SpecialMS_IndexPos_Batch_NMajor,
// the layout CIRBTS_BATCH_INDEX_NMAJOR=1 selects), into caller memory.
int ref_cirbts_index_nmajor(const uint64_t* d_a, uint32_t a_stride, uint32_t n, uint32_t batch, uint32_t N,
                            uint64_t q_lwe, uint32_t bitwidth, uint32_t* index_out, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    kernel_SpecialMS_IndexPos_Batch_NMajor<<<dim3((n + 255) / 256, batch), 256, 0, s>>>(d_a, index_out, n, batch, a_stride,
                                                                                        2 * N, q_lwe, bitwidth);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return static_cast<int>(e);
}

// Grouped (mb = 3) blind rotation in the configuration the reference's AES example selects by
// default for batched circuit bootstrapping (examples/aes_transcipher/main.cu:123-136:
// CIRBTS_PBS_MULTIBIT=3, CIRBTS_EVALACC_SOA=1, CIRBTS_BATCH_INDEX_NMAJOR=1, EvalAcc block X 128;
// fused-NTT threads per block from CIRBTS_FUSED_NTT_TPB, 384 in the AES fast defaults
// :107-121), launch sequence of bitwise/src/cirbts/cirbts-batch.cu:2640-2700: per group the INTT,
// kernel_SignedDigitDecompose2_FusedFNWT_Batch and kernel_EvalAccCore_Binary_MB3_Grouped_Batch_
// SoA_NMajor.  ek_soa / ek_shoup_soa: host arrays of the 7 subset keys ({0} {1} {2} {0,1} {0,2}
// {1,2} {0,1,2}), each in the SoA layout [groups][N/32 tiles][2 digits][2][32 lanes] with its
// Shoup table; index_nmajor from ref_cirbts_index_nmajor; ct [2 batch][N] and dct
// [2 digits batch][N] are caller scratch (nothing is allocated here, so a timed call measures
// the kernels only).  n must be a multiple of 3 (no tail group).
int ref_cirbts_blind_rotate_mb3_soa(uint64_t* acc, uint32_t n, uint32_t batch, const uint64_t* const* ek_soa,
                                    const uint64_t* const* ek_shoup_soa, const uint64_t* monic, const void* d_mod,
                                    const uint64_t* tw, const uint64_t* tws, const uint64_t* itw, const uint64_t* itws,
                                    const uint64_t* ninv, const uint64_t* ninv_s, uint32_t N, uint64_t Q,
                                    uint32_t base_g, uint32_t digits_g, const uint32_t* index_nmajor, uint32_t tpb,
                                    uint32_t block_x, uint64_t* ct, uint64_t* dct, void* stream) {
    if (n % 3 != 0 || tpb == 0 || block_x == 0) return static_cast<int>(cudaErrorInvalidValue);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const DModulus* mod = static_cast<const DModulus*>(d_mod);
    const uint32_t digitsG2 = 2 * digits_g, groups = n / 3, tiles = N / 32;
    const dim3 eb(block_x), eg((N + block_x - 1) / block_x, batch);
    cudaError_t e = cudaSuccess;
    for (uint32_t g = 0; g < groups && e == cudaSuccess; ++g) {
        inwt_1d_opt_outofplace_batched(ct, acc, itw, itws, mod, ninv, ninv_s, N, static_cast<size_t>(2) * batch, s);
        kernel_SignedDigitDecompose2_FusedFNWT_Batch<<<digitsG2 * batch, tpb, N * sizeof(uint64_t), s>>>(
            dct, ct, Q, base_g, digits_g, N, batch, tw, tws, mod);
        kernel_EvalAccCore_Binary_MB3_Grouped_Batch_SoA_NMajor<<<eg, eb, 0, s>>>(
            acc, dct, ek_soa[0], ek_shoup_soa[0], ek_soa[1], ek_shoup_soa[1], ek_soa[2], ek_shoup_soa[2], ek_soa[3],
            ek_shoup_soa[3], ek_soa[4], ek_shoup_soa[4], ek_soa[5], ek_shoup_soa[5], ek_soa[6], ek_shoup_soa[6], monic, N,
            tiles, mod, digitsG2, g, 3 * g, 3 * g + 1, 3 * g + 2, index_nmajor, batch);
        e = cudaGetLastError();
    }
    return static_cast<int>(e);
}

// HomTrace + SchemeSwitch of count MV RLWEs in the reference's default (unfused) launch
// sequence (bitwise/src/cirbts/cirbts-batch.cu:1656-1789): per round k the permuting INTT of
// c0, kernel_Fused_Permute_Decompose, the NTT of the digits and
// kernel_MultAddUpdate_HT_PermuteC1; kernel_SaveToRGSW of the trace (row 1); then INTT,
// decomposition, NTT and kernel_MultAddUpdate_SS against the s^2 key, saved as row 0.
// c0 / c1 [count][N] NTT domain (the MV RLWEs' two components), keys [rounds][digits_ht][2][N]
// and [digits_ss][2][N] with their Shoup tables, maps_out [rounds][N] receives the
// automorphism maps from the reference's kernel_GenerateCoefficientAutoMaps, rgsw_out
// [count][2 rows][2][N].  Returns the CUDA error code.
int ref_cirbts_trace_schemeswitch(const uint64_t* c0_in, const uint64_t* c1_in, uint32_t count, const uint64_t* ht_key,
                                  const uint64_t* ht_key_shoup, const uint64_t* ss_key, const uint64_t* ss_key_shoup,
                                  uint32_t rounds, uint32_t base_ht, uint32_t digits_ht, uint32_t base_ss,
                                  uint32_t digits_ss, uint32_t* maps_out, const void* d_mod, const uint64_t* tw,
                                  const uint64_t* tws, const uint64_t* itw, const uint64_t* itws, const uint64_t* ninv,
                                  const uint64_t* ninv_s, uint32_t N, uint64_t Q, uint64_t* rgsw_out, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const DModulus* mod = static_cast<const DModulus*>(d_mod);
    uint32_t logn = 0;
    while ((1u << logn) < N) ++logn;
    const size_t plane = static_cast<size_t>(count) * N;
    const uint32_t dmax = digits_ht > digits_ss ? digits_ht : digits_ss;
    uint64_t *c0 = nullptr, *c1 = nullptr, *n0 = nullptr, *n1 = nullptr, *perm = nullptr, *dig = nullptr, *s0 = nullptr,
             *s1 = nullptr;
    cudaError_t e = cudaSuccess;
    for (uint64_t** b : {&c0, &c1, &n0, &n1, &perm, &s0, &s1})
        if (e == cudaSuccess) e = cudaMalloc(b, sizeof(uint64_t) * plane);
    if (e == cudaSuccess) e = cudaMalloc(&dig, sizeof(uint64_t) * plane * dmax);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c0, c0_in, sizeof(uint64_t) * plane, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c1, c1_in, sizeof(uint64_t) * plane, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) {
        const dim3 block(256), grid((N + 255) / 256, count);
        kernel_GenerateCoefficientAutoMaps<<<dim3((N + 255) / 256, rounds), block, 0, s>>>(maps_out, N, logn, 2 * N - 1,
                                                                                            rounds);
        for (uint32_t k = 0; k < rounds; ++k) {
            const uint32_t* map = maps_out + static_cast<size_t>(k) * N;
            inwt_1d_opt_permute_batched(perm, c0, map, itw, itws, mod, ninv, ninv_s, N, count, s);
            kernel_Fused_Permute_Decompose<<<grid, block, 0, s>>>(dig, perm, Q, base_ht, digits_ht, N, count);
            fnwt_1d_opt_batched(dig, tw, tws, mod, N, static_cast<size_t>(count) * digits_ht, s);
            const size_t kofs = static_cast<size_t>(k) * digits_ht * 2 * N;
            kernel_MultAddUpdate_HT_PermuteC1<<<grid, block, 0, s>>>(n0, n1, dig, ht_key + kofs, ht_key_shoup + kofs, c0,
                                                                      c1, map, mod, digits_ht, N, count, plane);
            std::swap(c0, n0);
            std::swap(c1, n1);
        }
        kernel_SaveToRGSW<<<grid, block, 0, s>>>(rgsw_out, c0, c1, 1, N, count);
        inwt_1d_opt_batched(c0, itw, itws, mod, ninv, ninv_s, N, count, s);
        kernel_Fused_Permute_Decompose<<<grid, block, 0, s>>>(dig, c0, Q, base_ss, digits_ss, N, count);
        fnwt_1d_opt_batched(dig, tw, tws, mod, N, static_cast<size_t>(count) * digits_ss, s);
        kernel_MultAddUpdate_SS<<<grid, block, 0, s>>>(s0, s1, dig, ss_key, ss_key_shoup, c1, mod, digits_ss, N, count,
                                                        plane);
        kernel_SaveToRGSW<<<grid, block, 0, s>>>(rgsw_out, s0, s1, 0, N, count);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    for (uint64_t* b : {c0, c1, n0, n1, perm, dig, s0, s1}) cudaFree(b);
    return static_cast<int>(e);
}

}  // extern "C"
