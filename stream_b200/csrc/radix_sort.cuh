// Stable LSD radix sort of (u64 key, u32 value) pairs, "onesweep" style:
// one up-front histogram of every digit position, then one kernel per 8-bit
// digit that ranks a 4096-key tile with warp ballots, obtains its global
// offsets by decoupled look-back over earlier tiles, and scatters through
// shared memory so that global writes come out in digit runs.
//
// Replaces ava::sort::sort_pairs as used by LBVH::_sort_objects
// (include/geometry/lbvh.hpp:216-243): ascending keys, ties keep input order.
#pragma once

#include "common.cuh"

namespace sb {

constexpr int kSortBlock = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;  // 4096 keys per tile
constexpr int kSortMaxPasses = 8;

struct RadixSortPlan {
    DeviceBuffer<uint64_t> keys_alt;
    DeviceBuffer<uint32_t> vals_alt;
    DeviceBuffer<uint32_t> hist;      // [passes][256] counts, then exclusive digit offsets
    DeviceBuffer<uint32_t> lookback;  // [passes][tiles][256] flag|value words
    DeviceBuffer<uint32_t> tile_ctr;  // [passes] dynamic tile counters
    uint32_t tiles = 0;
    int passes = 0;

    // Size the scratch for n keys whose significant bits are [0, bits).
    void prepare(uint32_t n, int bits);
};

// Accumulate the digit histograms of one key into a shared [passes][256]
// table (used by the stand-alone histogram kernel and by producers that fuse
// it, such as the Morton-code kernel).
__device__ __forceinline__ void radix_hist_add(uint32_t* s_hist, uint64_t key, int passes) {
#pragma unroll
    for (int p = 0; p < kSortMaxPasses; ++p)
        if (p < passes) atomicAdd(&s_hist[p * 256 + (uint32_t)((key >> (8 * p)) & 0xffu)], 1u);
}

// Sort keys/vals of length n in place.  If hist_ready is true, plan.hist
// already holds the per-pass digit counts (fused producer); otherwise they are
// computed here.  Status bits are OR-ed into d_status on look-back timeout.
void radix_sort_pairs(RadixSortPlan& plan, uint64_t* keys, uint32_t* vals, uint32_t n, int bits,
                      bool hist_ready, uint32_t* d_status, cudaStream_t stream);

}  // namespace sb
