// Device-wide exclusive scan of u32 counts into n+1 offsets (out[0] = 0,
// out[n] = total), replacing ava::scan::inclusive_sum at
// src/mesh/DirectAlphaShape3D.cpp:235-249,697-704 (which write row offsets
// shifted by one).  Reduce-then-scan over 4096-element tiles.
#pragma once

#include "common.cuh"

namespace sb {

struct ScanPlan {
    DeviceBuffer<uint32_t> partial;
};

void exclusive_scan_u32(ScanPlan& plan, const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t stream);

}  // namespace sb
