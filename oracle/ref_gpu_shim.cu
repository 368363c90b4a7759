// ref_gpu_shim.cu -- C entry points around the reference's own Phantom NTT kernels
// (src/ntt/ntt_1d.cu, src/ntt/fntt_2d.cu, src/ntt/intt_2d.cu), compiled for sm_100a from the
// reference sources by `make -C oracle ref_gpu`.  Test and measurement infrastructure only:
// the GPU tests use it as a second parity check of the product's NTTs, and bench.py times it
// beside the product's kernels as the reference's GPU baseline on the same B200.  Nothing in
// the product loads it.
#include <cstdint>
#include <vector>

#include "ntt.cuh"

using phantom::arith::Modulus;
using phantom::arith::NTT;

extern "C" {

// fnwt_1d_opt_batched (include/ntt.cuh:215): in place, dim in {2048, 4096} per the kernel's
// one-block design, tables as produced by phantom::arith::NTT
int ref_gpu_fnwt_1d_opt_batched(uint64_t* inout, const uint64_t* tw, const uint64_t* tws, const void* mod,
                                size_t dim, size_t batch, void* stream) {
    fnwt_1d_opt_batched(inout, tw, tws, static_cast<const DModulus*>(mod), dim, batch,
                        static_cast<cudaStream_t>(stream));
    return static_cast<int>(cudaGetLastError());
}

// inwt_1d_opt_batched (include/ntt.cuh:219)
int ref_gpu_inwt_1d_opt_batched(uint64_t* inout, const uint64_t* itw, const uint64_t* itws, const void* mod,
                                const uint64_t* scalar, const uint64_t* scalar_shoup, size_t dim, size_t batch,
                                void* stream) {
    inwt_1d_opt_batched(inout, itw, itws, static_cast<const DModulus*>(mod), scalar, scalar_shoup, dim, batch,
                        static_cast<cudaStream_t>(stream));
    return static_cast<int>(cudaGetLastError());
}

// DNTTTable of a modulus chain (the constructor of include/ntt.cuh:127-150), built from the
// reference's host NTT class
void* ref_gpu_ntt2d_create(uint32_t log_n, uint32_t size, const uint64_t* h_q) {
    const uint64_t n = uint64_t(1) << log_n;
    std::vector<DModulus> dm(size);
    std::vector<uint64_t> tw(n * size), tws(n * size), itw(n * size), itws(n * size), ni(size), nis(size);
    for (uint32_t i = 0; i < size; ++i) {
        const Modulus m(h_q[i]);
        const NTT t(static_cast<int>(log_n), m);
        dm[i] = DModulus(m.value(), m.const_ratio()[0], m.const_ratio()[1]);
        for (uint64_t k = 0; k < n; ++k) {
            tw[i * n + k] = t.get_from_root_powers()[k];
            tws[i * n + k] = t.get_from_root_powers_shoup()[k];
            itw[i * n + k] = t.get_from_inv_root_powers()[k];
            itws[i * n + k] = t.get_from_inv_root_powers_shoup()[k];
        }
        ni[i] = t.inv_degree_modulo();
        nis[i] = t.inv_degree_modulo_shoup();
    }
    auto* table = new DNTTTable(n, size, dm.data(), tw.data(), tws.data(), itw.data(), itws.data(), ni.data(),
                                nis.data(), cudaStreamLegacy);
    cudaStreamSynchronize(cudaStreamLegacy);
    return table;
}

int ref_gpu_ntt2d_forward(void* table, uint64_t* inout, uint32_t coeff_modulus_size, uint32_t start_modulus_idx,
                          void* stream) {
    nwt_2d_radix8_forward_inplace(inout, *static_cast<DNTTTable*>(table), coeff_modulus_size, start_modulus_idx,
                                  static_cast<cudaStream_t>(stream));
    return static_cast<int>(cudaGetLastError());
}

int ref_gpu_ntt2d_backward(void* table, uint64_t* inout, uint32_t coeff_modulus_size, uint32_t start_modulus_idx,
                           void* stream) {
    nwt_2d_radix8_backward_inplace(inout, *static_cast<DNTTTable*>(table), coeff_modulus_size, start_modulus_idx,
                                   static_cast<cudaStream_t>(stream));
    return static_cast<int>(cudaGetLastError());
}

void ref_gpu_ntt2d_destroy(void* table) {
    cudaDeviceSynchronize();
    delete static_cast<DNTTTable*>(table);
}

}  // extern "C"
