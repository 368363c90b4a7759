// host_math.h -- host-side number theory for table construction (product code).
//
// Restates Phantom's host routines: get_primes (src/host/numth.cu:207-233),
// try_minimal_primitive_root (src/host/numth.cu:309-331) and the NTT table layout of
// phantom::arith::NTT (src/host/ntt.cu:11-56).  Exact unsigned __int128 arithmetic.
#pragma once

#include <cstdint>
#include <vector>

namespace cbs {
namespace host {

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q);
uint64_t powmod(uint64_t a, uint64_t e, uint64_t q);
uint64_t invmod(uint64_t a, uint64_t q);
uint64_t shoup(uint64_t w, uint64_t q);
bool is_prime(uint64_t n);
bool get_primes(uint32_t ntt_size, int bit_size, uint32_t count, std::vector<uint64_t>& out);
uint64_t minimal_primitive_root(uint64_t degree, uint64_t q);
uint32_t bit_reverse(uint32_t x, int bits);
void barrett_ratio(uint64_t q, uint64_t& r0, uint64_t& r1);

struct NttTables {
    uint32_t n = 0;
    uint64_t q = 0;
    std::vector<uint64_t> rp, rp_sh, irp, irp_sh;
    uint64_t n_inv = 0, n_inv_sh = 0;
    uint64_t ratio0 = 0, ratio1 = 0;
    uint64_t root = 0;
};

bool make_ntt_tables(uint32_t n, uint64_t q, NttTables& t);

// exact host negacyclic NTT with the same tables (used only by host-side key setup)
void ntt_forward_host(uint64_t* a, const NttTables& t);
void ntt_inverse_host(uint64_t* a, const NttTables& t);

}  // namespace host
}  // namespace cbs
