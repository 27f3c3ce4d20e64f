// 3D "direct" alpha shape on B200: per-point star Delaunay with exact
// predicates, alpha filter, free-surface flags and CSR output.
//
// Mirrors stream::mesh::AlphaShape3D (include/mesh/DirectAlphaShape3D.hpp:
// 73-305, src/mesh/DirectAlphaShape3D.cpp:121-743).  Output ids are Morton
// ordered like the reference's (use `perm` to map back: point i of the
// Morton order is input point perm[i]).
//
// Layout in HBM (N points, W = ceil(N/32) warp blocks):
//   obj_m   float4[N+4]        Morton-ordered (x, y, z, alpha) + 4 infinity points
//   cand    u32[W][124][32]    candidate neighbours, lane-interleaved so a warp
//                              reading entry j of its 32 stars is one 128 B line
//   tets    u32[W][252][32]    local tets (3 local ids packed in a word), same
//   nineig  u32[N]             star size incl. the 4 infinity ids (<= 128)
//   emask   uint4[N]           local ids used by a kept tet (edge present)
//   bmask   uint4[N]           ... used by at most 3 kept tets (boundary edge)
//   nout/nfneig u32[N], nkeep/node_is_bnd u8[N]
//   elemrow/row u32[N+1], elems uint4[n_elems], neig u32[n_edges], edge_is_bnd u8[n_edges]
// The star is capped at 128 local ids (124 neighbours in traversal order),
// as in the reference (DirectAlphaShape3D.cpp:362-363); the cap bounds the
// per-point storage at 1.5 KB whatever the candidate count.
#pragma once

#include "common.cuh"
#include "lbvh.cuh"
#include "scan.cuh"

namespace sb {

constexpr int kStarCap = 128;               // local ids incl. 4 infinity points
constexpr int kCandMax = kStarCap - 4;       // 124
constexpr int kTetCap = 2 * kCandMax + 4;    // 252 = 2V - 4 for V = 128

// Placement of the per-star candidate and tet lists: entry j of star s is at
// list_base<kI, kCap>(s) + j * kI.  kI = 32 interleaves 32 consecutive stars
// (entry j of a warp's 32 stars in one 128-byte line); kI = 1 keeps each
// star's list contiguous.
#ifndef SB_CAND_INTERLEAVE
#define SB_CAND_INTERLEAVE 32
#endif
#ifndef SB_TET_INTERLEAVE
#define SB_TET_INTERLEAVE 32
#endif
constexpr uint32_t kCandInterleave = SB_CAND_INTERLEAVE;
constexpr uint32_t kTetInterleave = SB_TET_INTERLEAVE;
template <uint32_t kI, uint32_t kCap>
__host__ __device__ __forceinline__ size_t list_base(uint32_t s) {
    return (size_t)(s / kI) * kCap * kI + (s % kI);
}
__host__ __device__ __forceinline__ size_t cand_at(uint32_t s, uint32_t j) {
    return list_base<kCandInterleave, kCandMax>(s) + (size_t)j * kCandInterleave;
}

struct AlphaShape3D : LBVH3D::StageMarks {
    uint32_t n_nodes = 0, n_elems = 0, n_edges = 0;
    int bits = 63;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t own_stream_saved = nullptr;

    DeviceBuffer<float4> nodes;  // input spheres
    LBVH3D lbvh;
    DeviceBuffer<uint32_t> cand, tets, nineig, nout, nfneig;
    DeviceBuffer<uint8_t> nkeep, node_is_bnd;
    DeviceBuffer<uint4> emask, bmask;
    DeviceBuffer<uint32_t> elemrow, row, neig;
    DeviceBuffer<uint4> elems;
    DeviceBuffer<uint8_t> edge_is_bnd;
    DeviceBuffer<uint32_t> words;     // [0] status bits [1] deferred stars [2] truncated [3] exact calls
    DeviceBuffer<uint32_t> deferred;  // stars queued for the exact pass: {star, stop state} pairs
    ScanPlan scan;
    PinnedWords pinned;
    DeviceBuffer<float> staging;      // host-input staging (coords then alpha)
    DeviceBuffer<uint32_t> input_bad; // set when the staged input holds an infinite or NaN value

    // Optional per-stage device timing (CUDA events on the handle's stream).
    enum Stage { S_BBOX_MORTON, S_SORT, S_GATHER_KARRAS_FIT, S_CANDIDATES, S_STAR, S_STAR_EXACT, S_SCAN, S_COMPRESS,
                 S_COUNT };
    bool profiling = false;
    cudaEvent_t ev[S_COUNT + 1] = {};
    float stage_ms[S_COUNT] = {};
    void mark(int i);                 // record event i when profiling
    void collect_profile();
    void mark_sort() override { mark(S_SORT); }
    void mark_gather() override { mark(S_GATHER_KARRAS_FIT); }
    uint32_t last_status = 0, last_truncated = 0, last_exact = 0, last_deferred = 0;
    // Work counters of the fast star pass (stage-1 insphere tests, stage-2
    // FP64 evaluations), filled by compute() while count_work is set.
    bool count_work = false;
    DeviceBuffer<unsigned long long> work;
    bool inited = false, computed = false;

    AlphaShape3D();
    virtual ~AlphaShape3D();

    // Host arrays: coords N x 3 row-major, alpha N (DirectAlphaShape3D.cpp:764-777).
    void set_nodes_host(uint32_t n, const float* coords, const float* alpha);
    // Device spheres (x, y, z, alpha), N entries.
    void set_nodes_device(uint32_t n, const float4* spheres);
    // LBVH build, infinity points and the candidate-neighbour pass.
    void init();
    // Star Delaunay + alpha filter + scans + compress (= compute() + compress()).
    void compute();
    // Synchronise and refresh the counters (status, truncated, exact, deferred).
    void read_counters();
    // Run on a caller-owned stream (nullptr: back to the handle's own stream).
    void set_stream(cudaStream_t s);
};

// Evaluate the star kernel's conflict decision for m point quintuples on the
// device (test entry; synchronous).
void conflict_batch_device(uint32_t m, const float* d_pts, const uint32_t* d_ids, float* d_out, uint32_t* d_status,
                           cudaStream_t stream);

}  // namespace sb
