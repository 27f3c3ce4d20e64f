// Karras LBVH over 3D spheres (x, y, z, r as float4), B200-native.
//
// Mirrors stream::geo::LBVH<Sphere3D, DataF, 3>::build
// (include/geometry/lbvh.hpp:354-360): global box (:141-175), Morton codes
// (:178-213), stable sort + gather (:216-243), Karras hierarchy (:246-308)
// and bottom-up boxes (:311-351).  Arrays keep the reference's meaning so
// results can be compared bit for bit: codes/perm after the sort, sep (the
// split gamma of internal node i), cil (bit 0: left child is a leaf, bit 1:
// right child is a leaf), parents with bit 31 marking a right child, and one
// box per internal node (node 0 is the root).
#pragma once

#include "common.cuh"
#include "radix_sort.cuh"

namespace sb {

struct NodeBox {  // internal-node box, 32 B so a child pair is one 64 B line
    float4 lo;  // x, y, z, unused
    float4 hi;
};

struct LBVH3D {
    uint32_t n = 0;
    int bits = 63;           // 63 (21 bits per axis, the reference), 30 (10 bits per axis) or
                             // 64: 2D points (x, y, unused, r), 32 bits per axis (dim = 2)
    bool fit_point = false;  // leaf box = centre only (alpha shape) instead of sphere box
    uint32_t tail = 0;       // extra float4 slots reserved after obj_m (alpha-shape infinity points)

    DeviceBuffer<float4> obj_m;       // n (+tail) spheres in Morton order
    DeviceBuffer<uint64_t> codes;     // n sorted codes
    DeviceBuffer<uint32_t> perm;      // n: obj_m[i] = obj[perm[i]] (getPermutation)
    DeviceBuffer<int32_t> sep;        // n-1
    DeviceBuffer<uint8_t> cil;        // n-1
    DeviceBuffer<uint32_t> leaf_parent;      // n
    DeviceBuffer<uint32_t> internal_parent;  // n-1
    DeviceBuffer<uint32_t> touched;          // n-1
    DeviceBuffer<NodeBox> boxes;             // n-1
    DeviceBuffer<float> bb_glob;             // 6: pmin, pmax (includes the radii)
    DeviceBuffer<int> bb_enc;                // 6 ordered-int encodings for atomics
    RadixSortPlan sort;

    // Build from n device spheres.  d_status collects status bits.  `prof`
    // (may be null) receives stage marks: sort start, gather start, hierarchy start.
    struct StageMarks {
        virtual void mark_sort() = 0;
        virtual void mark_gather() = 0;
        virtual void mark_hierarchy() {}  // before the Karras hierarchy (build() only)
    };
    void build(const float4* d_obj, uint32_t n, cudaStream_t stream, uint32_t* d_status, StageMarks* prof = nullptr);
    // First half of build(): global box, Morton codes, sort, gather into
    // obj_m.  Shared with the TRBVH, whose codes are the same (trbvh.hpp:209-243).
    void sort_stage(const float4* d_obj, uint32_t n, cudaStream_t stream, uint32_t* d_status, StageMarks* prof);
};

}  // namespace sb
