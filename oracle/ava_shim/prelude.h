// Force-included (g++ -include) before every reference translation unit that
// the oracle build compiles.  Maps the host clz builtin onto a version that is
// defined at zero (64, as on CUDA), which the reference's Karras build relies
// on for duplicate Morton codes (include/geometry/lbvh.hpp:257-258,273,279).
#pragma once
#include "ava_shim.hpp"
#define __builtin_clzll(x) ava_shim_clzll(x)
