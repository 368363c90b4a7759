// Stand-in for OpenFHE's lwe-keyswitchkey.h when the reference's bitwise/examples/
// aes_gpu_ks.cuh is compiled alone: a switching key whose GetElementsA()[i][v][j][k] /
// GetElementsB()[i][v][j] have ConvertToInt(), the shape that header's key packing reads.
// Test infrastructure.
#pragma once

#include <memory>
#include <vector>

#include "lwe-cryptoparameters.h"

namespace lbcrypto {

struct ShimLWESwitchingKey {
    std::vector<std::vector<std::vector<std::vector<ShimNativeInteger>>>> a;
    std::vector<std::vector<std::vector<ShimNativeInteger>>> b;
    const decltype(a)& GetElementsA() const { return a; }
    const decltype(b)& GetElementsB() const { return b; }
};
using ConstLWESwitchingKey = std::shared_ptr<const ShimLWESwitchingKey>;

}  // namespace lbcrypto
