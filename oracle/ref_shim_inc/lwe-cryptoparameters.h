// Stand-in for OpenFHE's lwe-cryptoparameters.h (the absent OpenFHE fork) when the reference's
// bitwise/examples/aes_gpu_ks.cuh is compiled alone: BasicInteger and the four accessors of
// LWECryptoParams that header's host helpers read.  Test infrastructure.
#pragma once

#include <cstdint>

typedef uint64_t BasicInteger;

namespace lbcrypto {

struct ShimNativeInteger {
    uint64_t v = 0;
    uint64_t ConvertToInt() const { return v; }
};

class LWECryptoParams {
public:
    ShimNativeInteger GetqKS() const { return qks; }
    uint32_t GetBaseKS() const { return base_ks; }
    uint32_t Getn() const { return n; }
    uint32_t GetN() const { return N; }
    ShimNativeInteger qks;
    uint32_t base_ks = 0, n = 0, N = 0;
};

}  // namespace lbcrypto
