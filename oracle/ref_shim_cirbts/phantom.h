// Stand-in for the reference's umbrella "phantom.h" when its CirBTS kernels are compiled alone:
// only the Phantom headers those kernels use (DModulus and the NTT entry points, the modular
// butterflies), not the CKKS context headers that pull in OpenFHE.  Test infrastructure.
#pragma once

#include <cuda_runtime.h>

#include "butterfly.cuh"
#include "ntt.cuh"
