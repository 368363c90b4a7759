// ref_gpu_extract_shim.cu -- C entry point around the reference's own sample-extract + LWE
// key-switch kernel (kernel_SampleExtractKeySwitchToLWE, bitwise/examples/aes_gpu_ks.cuh:
// 538-607, with its launch helpers :696-760), compiled for sm_100a from the reference header
// where it lies by `make -C oracle ref_gpu_extract`, with the stand-in headers of
// ref_shim_inc/ for the OpenFHE and Phantom headers it includes.  Test infrastructure only:
// the GPU tests run it beside cbs_extract_keyswitch_device on the same words and key.
#include <cstdint>

#include "phantom.h"
#include "lwe-cryptoparameters.h"
#include "lwe-keyswitchkey.h"
#include "aes_gpu_ks.cuh"

extern "C" {

// d_ksk [2][N][base_ks][n+1] u16 (the packed layout of GpuLweKeySwitchKeyU16::TryInit);
// d_rlwe_a / d_rlwe_b [words][N] coefficient domain mod Q; d_info[count] = (word << 16) | idx;
// outputs d_out_a [count][out_stride], d_out_b [count] mod q_lwe.  mapped != 0 selects the
// pre-encoded coefficient-map variant.  The constants follow the reference's caller
// (aes_transcipher/extract.cuh:226-234).  Returns 0 on success.
int ref_gpu_extract_keyswitch(const uint16_t* d_ksk, uint32_t n, uint32_t N, uint32_t base_ks, uint32_t qks,
                              const uint64_t* d_rlwe_a, const uint64_t* d_rlwe_b, const uint32_t* d_info,
                              uint32_t count, uint64_t Q, uint64_t q_lwe, uint64_t* d_out_a, uint64_t* d_out_b,
                              uint32_t out_stride, int mapped) {
    try {
        aes_example::GpuLweKeySwitchKeyU16 key;
        key.d_ksk = const_cast<uint16_t*>(d_ksk);
        key.n = n;
        key.N = N;
        key.baseKS = base_ks;
        key.baseKS_log2 = aes_example::Log2Pow2(base_ks);
        key.digitCount = aes_example::DigitCountPow(qks, base_ks);
        key.qKS = qks;
        key.qKS_mask = qks - 1u;
        key.elems = static_cast<size_t>(key.digitCount) * N * base_ks * (n + 1);
        bool ok = false;
        {
            aes_example::GpuLweKeySwitchWorkspaceU16 ws(count, N, n);
            const double q_over_Q = static_cast<double>(qks) / static_cast<double>(Q);
            const bool q_divisible = (q_lwe % qks) == 0;
            const uint64_t scale = q_divisible ? (q_lwe / qks) : 0;
            if (mapped)
                ok = aes_example::KeySwitchBatchDeviceFromMappedExtractedRLWEToLWE(
                    key, ws, d_rlwe_a, d_rlwe_b, d_info, d_out_a, d_out_b, count, Q, q_over_Q, q_divisible, scale,
                    q_lwe, out_stride);
            else
                ok = aes_example::KeySwitchBatchDeviceFromExtractedRLWEToLWE(
                    key, ws, d_rlwe_a, d_rlwe_b, d_info, d_out_a, d_out_b, count, Q, q_over_Q, q_divisible, scale,
                    q_lwe, out_stride);
            if (ok) PHANTOM_CHECK_CUDA(cudaStreamSynchronize(ws.stream));
        }
        key.d_ksk = nullptr;  // the caller owns the key buffer
        return ok ? 0 : 1;
    } catch (...) {
        return 2;
    }
}

}  // extern "C"
