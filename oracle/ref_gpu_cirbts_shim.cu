// ref_gpu_cirbts_shim.cu -- drives the reference's own one-bit GINX blind-rotation kernels,
// compiled for sm_100a from bitwise/src/cirbts/kernel.cu and src/ntt/ntt_1d.cu where they lie
// (`make -C oracle ref_gpu_cirbts`, stand-in headers in ref_shim_cirbts/), in the launch
// sequence of the reference's batched blind rotation (bitwise/src/cirbts/cirbts-batch.cu:
// 3438-3446 index positions, 4064-4075 per-step INTT + fused decomposition/NTT, 3976-3980
// binary MAC with the AoS key).  Test infrastructure only: the GPU tests compare the
// accumulator it produces with the oracle's, which the product's NTT path matches bit for bit.
#include <cstdint>
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

}  // extern "C"
