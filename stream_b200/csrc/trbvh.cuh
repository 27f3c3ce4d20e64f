// TRBVH over 3D spheres on B200: Apetrei agglomerative build over the sorted
// Morton codes, then Karras-Aila treelet restructuring rounds.
//
// Mirrors stream::geo::TRBVH<Sphere3D, ComputeBB_Functor<Sphere3D>, 3>
// (include/geometry/trbvh.hpp:65-681).  Node ids: leaves 0..n-1 (Morton
// order), internal nodes n..2n-2, root parent 2n.  The Apetrei topology,
// ranges, boxes and subtree sizes equal the reference's.  The SAH cost is
// order independent (cost(leaf) = Ct A, cost(node) = (Ci A + cost(l)) +
// cost(r)) instead of the reference's arrival-order accumulation
// (trbvh.hpp:326-373), which makes the restructured tree deterministic.
// Treelet size (default 7; the reference fixes 5) and the area measure (3D
// half surface xy+yz+zx by default; the reference's ext_x*ext_y as an option)
// are parameters.
#pragma once

#include "common.cuh"
#include "lbvh.cuh"

namespace sb {

constexpr int kTreeletMax = 8;

struct TRBVH3D {
    uint32_t n = 0;
    int treelet_size = 7;
    bool area3d = true;
    int rounds = 3;

    LBVH3D sorter;  // box, Morton codes, sort, gather (obj_m, codes, perm)
    DeviceBuffer<uint32_t> child_left, child_right, range_min, range_max;  // n-1
    DeviceBuffer<uint32_t> parent, subtree_size;                           // 2n-1
    DeviceBuffer<NodeBox> boxes;                                           // 2n-1
    DeviceBuffer<float> sah;                                               // 2n-1
    DeviceBuffer<uint64_t> delta;                                          // n-1
    DeviceBuffer<uint32_t> touched;                                        // n-1
    DeviceBuffer<uint32_t> root;                                           // 1

    // prof (may be null): sort and gather marks from the shared sort stage,
    // then mark_hierarchy() before the Apetrei build; mark_treelets() before
    // the restructuring rounds.
    struct StageMarks : LBVH3D::StageMarks {
        virtual void mark_treelets() {}
    };
    void build(const float4* d_obj, uint32_t n, cudaStream_t stream, uint32_t* d_status, StageMarks* prof = nullptr);
    // Per object, the number of other objects whose sphere overlaps its own
    // (depth-first search of the tree; tests/geometry/trbvh_random_collision.cpp).
    void count_overlaps(uint32_t* d_out, cudaStream_t stream) const;
};

}  // namespace sb
