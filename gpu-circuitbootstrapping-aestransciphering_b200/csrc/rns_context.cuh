// rns_context.cuh -- the cbs_rns_context object behind the RNS (Phantom-core) C ABI, shared by
// rns.cu (NTT entry points, modup / inner product / moddown / keyswitch) and ckks.cu (the CKKS
// evaluator operations built on them).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <vector>

#include "../../include/cbs_b200.h"
#include "devbuf.cuh"
#include "host_math.h"
#include "ntt_rns.cuh"

namespace cbs {

// per-level constants of modup / moddown (built on first use of a level)
struct RnsLevel {
    uint32_t ql = 0, qlp = 0, alpha = 0, beta = 0, ntt_limbs = 0;
    DevBuf<uint64_t> mu_scale, mu_scale_s;       // [ql] partQlHatInv_mod_Ql (rns.cu:120-200)
    DevBuf<uint32_t> mu_out_slot, mu_out_prime;  // [beta][qlp] complement limbs of each digit
    DevBuf<uint64_t> mu_qhat;                    // [beta][qlp][alpha] qhat_i mod m_out
    DevBuf<uint32_t> mu_ntt_slot, mu_ntt_prime;  // [ntt_limbs] limbs transformed after bconv
    DevBuf<uint32_t> ip_prime;                   // [qlp] key-chain index of limb l of QlP
    DevBuf<uint32_t> md_slot, md_prime;          // [alpha] P limbs inside a QlP poly
    DevBuf<uint64_t> md_scale, md_scale_s;       // [alpha] Phat_j^-1 mod p_j
    DevBuf<uint64_t> md_phat;                    // [ql][alpha] Phat_j mod q_i
    DevBuf<uint64_t> md_pinv, md_pinv_s;         // [ql] P^-1 mod q_i
};

}  // namespace cbs

struct cbs_rns_context {
    uint32_t log_n = 0, n = 0, size_q = 0, size_p = 0, size_qp = 0;
    uint32_t red_k = 1;
    int device = 0;
    std::vector<uint64_t> primes;  // Q chain then P
    std::vector<cbs::host::NttTables> tabs;
    cbs::DevBuf<uint64_t> d_tw, d_tws, d_itw, d_itws, d_q, d_ninv, d_ninv_s, d_r0, d_r1;
    cbs::DevBuf<double> d_twd, d_itwd;  // tw / itw as doubles when every prime is below 2^50
    cbs::DevBuf<double> d_qinv;         // fl(1 / q) per prime, likewise
    cbs::DevBuf<uint32_t> d_fault;      // device fault word (CBS_FAULT_* bits)
    cbs::DevBuf<cbs_dmodulus> d_mod;
    cbs::DevBuf<uint32_t> d_ident;  // 0 .. size_qp - 1
    std::map<uint32_t, std::unique_ptr<cbs::RnsLevel>> levels;
    cbs::DevBuf<uint64_t> s_coef, s_t, s_cx, s_delta;  // scratch, grown on demand
    // CKKS evaluator (ckks.cu): scratch, q_last^-1 tables per level, Galois slot permutations
    cbs::DevBuf<uint64_t> s_ck0, s_ck1;
    std::map<uint32_t, std::unique_ptr<cbs::DevBuf<uint64_t>>> rescale_tab;
    std::map<uint32_t, std::unique_ptr<cbs::DevBuf<uint32_t>>> galois_perm;

    cbs::RnsNttArgs ntt_args() const {
        cbs::RnsNttArgs a;
        a.tw = d_tw.p;
        a.tws = d_tws.p;
        a.itw = d_itw.p;
        a.itws = d_itws.p;
        a.q = d_q.p;
        a.n_inv = d_ninv.p;
        a.n_inv_s = d_ninv_s.p;
        a.twd = d_twd.p;
        a.itwd = d_itwd.p;
        a.fault = d_fault.p;
        return a;
    }
};

namespace cbs {

// level constants of size_ql (built once, on first use)
cbs_status build_level(cbs_rns_context* c, uint32_t ql, RnsLevel** out);
// size_ql within [1, size_q]
cbs_status check_level(const cbs_rns_context* c, uint32_t size_ql);
// grow a scratch buffer to at least `words`
cbs_status grow(DevBuf<uint64_t>& b, size_t words);
// keyswitch of count ciphertexts: d_ct [count][2][ql][N] += KS(d_c2 [count][ql][N])
cbs_status run_keyswitch(cbs_rns_context* c, uint64_t* d_ct, const uint64_t* d_c2, const uint64_t* const* h_evks,
                         uint32_t size_ql, uint32_t count, cudaStream_t s);

}  // namespace cbs
