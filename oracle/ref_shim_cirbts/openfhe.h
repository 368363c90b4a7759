// Stand-in for OpenFHE's umbrella header (the absent OpenFHE fork) when the reference's
// CirBTS kernels (bitwise/src/cirbts/kernel.cu) are compiled alone: the two integer types those
// kernels use.  Test infrastructure.
#pragma once

#include <cstdint>

typedef uint64_t BasicInteger;

namespace lbcrypto {
struct NativeInteger {
    typedef int64_t SignedNativeInt;
};
}  // namespace lbcrypto
using lbcrypto::NativeInteger;
