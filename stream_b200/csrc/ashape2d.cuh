// 2D "direct" alpha shape on B200: per-point star Delaunay (a fan of
// triangles around the point) with exact predicates, alpha filter, boundary
// flags and CSR output.
//
// Mirrors stream::mesh::AlphaShape2D (include/mesh/DirectAlphaShape2D.hpp:
// 74-345, src/mesh/DirectAlphaShape2D.cpp:121-690).  Output ids are Morton
// ordered like the reference's (point i of the Morton order is input point
// perm[i]).
//
// Layout in HBM (N points, W = ceil(N/32) warp blocks, L_w = 3 + the largest
// neighbour count in block w, from the count pass):
//   obj_m   float4[N+3]          Morton-ordered (x, y, 0, alpha) + 3 infinity points
//   boff    u32[W+1]             block offsets: boff[w+1] - boff[w] = 32 L_w
//   cand    u32[boff[W]]         global id of local id a of point 32w+l at
//                                boff[w] + 32a + l (lane-interleaved: a warp
//                                reading the same a of its 32 stars is one line);
//                                ids 0..2 are the infinity points, then the
//                                neighbours in traversal order
//   ccoord  float2[boff[W]]      their coordinates, same layout (the star loop
//                                reads one 8-byte word per vertex)
//   act     u8[boff[W]]          kept triangles per local id (edge present /
//                                boundary edge when 1), same layout
//   tris    u32[boff[W]]         local triangles (a | b << 8 | orientation sign
//                                << 16), same layout: a star of L local ids has
//                                at most L triangles
//   nineig  u32[N]               star size incl. the 3 infinity ids (<= 252)
//   nout/nfneig u32[N], nkeep/node_is_bnd u8[N]
//   elemrow/row u32[N+1], elems u32[3 n_elems], neig u32[n_edges], edge_is_bnd u8[n_edges]
// The fill pass keeps the reference's limit: it stops once a point holds more
// than 250 local ids (DirectAlphaShape2D.cpp:351-354).
#pragma once

#include "common.cuh"
#include "lbvh.cuh"
#include "scan.cuh"

namespace sb {

constexpr uint32_t kInf2 = 3;          // infinity points (DirectAlphaShape2D.hpp:101)
constexpr uint32_t kFillLimit2 = 250;  // fill-pass stop (DirectAlphaShape2D.cpp:351)

struct AlphaShape2D : LBVH3D::StageMarks {
    uint32_t n_nodes = 0, n_elems = 0, n_edges = 0;
    size_t slots = 0;  // boff[W]
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t own_stream_saved = nullptr;

    DeviceBuffer<float4> nodes;  // input (x, y, 0, alpha)
    LBVH3D lbvh;                 // bits = 64: the 2D Morton code
    DeviceBuffer<uint32_t> bsz, boff, cand, nineig, nout, nfneig;
    DeviceBuffer<float2> ccoord;
    DeviceBuffer<uint8_t> act, nkeep, node_is_bnd;
    DeviceBuffer<uint32_t> tris;
    DeviceBuffer<uint32_t> elemrow, row, neig, elems;
    DeviceBuffer<uint8_t> edge_is_bnd;
    DeviceBuffer<uint32_t> words;  // [0] status bits [1] stars stopped at the fill limit [2] exact in-circle calls
                                   // [6] star work queue
    ScanPlan scan;
    PinnedWords pinned;
    DeviceBuffer<float> staging;
    DeviceBuffer<uint32_t> input_bad;  // set when the staged input holds an infinite or NaN value

    enum Stage { S_LBVH, S_COUNT_PASS, S_FILL, S_STAR, S_SCAN, S_COMPRESS, S_COUNT };
    bool profiling = false;
    cudaEvent_t ev[S_COUNT + 1] = {};
    float stage_ms[S_COUNT] = {};
    void mark(int i);
    void collect_profile();
    void mark_sort() override {}
    void mark_gather() override {}
    uint32_t last_status = 0, last_limited = 0, last_exact = 0;
    bool inited = false, computed = false;

    AlphaShape2D();
    virtual ~AlphaShape2D();

    // Host arrays: coords N x 2 row-major, alpha N (DirectAlphaShape2D.cpp:708-721).
    void set_nodes_host(uint32_t n, const float* coords, const float* alpha);
    // Device points (x, y, unused, alpha), N entries.
    void set_nodes_device(uint32_t n, const float4* pts);
    // LBVH build, infinity points, neighbour count pass and the ELL layout
    // (AlphaShape2D::init, DirectAlphaShape2D.cpp:121-290).
    void init();
    // Fill pass, star Delaunay + alpha filter, scans and compress
    // (AlphaShape2D::compute + compress, :293-690).
    void compute();
    void read_counters();
    void set_stream(cudaStream_t s);
};

}  // namespace sb
