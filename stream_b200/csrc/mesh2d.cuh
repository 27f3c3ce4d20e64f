// 2D Delaunay triangulation on B200 behind the reference's Mesh2D interface
// (include/mesh/mesh.hpp, src/mesh/mesh.cpp:818-862): the triangulation of
// the points and three super nodes, whose triangles are dropped by
// remove_super_nodes.
//
// Each point owns its star (the fan of Delaunay triangles around it), built
// by incremental insertion with the 2D alpha-shape star kernel's conflict
// predicate (FP32 in-circle filter, exact expansion, Simulation of
// Simplicity), so that all stars decide every in-circle question the same
// way.  A star triangle is *verified* once a query of the point LBVH finds no
// point strictly inside its circumcircle: verified triangles are Delaunay in
// the whole point set and are never removed again.  A query that finds a
// point inserts it into the star.  A star whose triangles are all verified is
// the point's star in the Delaunay triangulation of points + super nodes, so
// the owner-compressed stars (each triangle written by its smallest id) form
// that triangulation.
//
// Phases (the reference's names):
//   init                     LBVH over the points (Morton order), super nodes,
//                            each star = the three super triangles
//   insert_morton_neighbors  insert the kMortonSeed points before and after
//                            each point in Morton order
//   insert_BVH_neighbors     one verification sweep (at most one query per
//                            triangle present when the sweep starts)
//   insert_iterative         verify until every triangle is verified
//   remove_super_nodes       leave triangles with a super node out of the output
//
// Layout in HBM (N points, lane-interleaved by warps of 32 stars: local slot a
// of point i at (i / 32) * 32 * kLocal2 + 32 a + i % 32):
//   obj_m   float4[N+3]       Morton-ordered (x, y, 0, 0) + the 3 super nodes
//   loc     u32[32 W kLocal2] global id of each local id (0..2: super nodes)
//   tri     u32[32 W kLocal2] star triangles a | b << 8 | (orient2d < 0) << 16
//                             | verified << 17 (a, b local ids)
//   nloc, ntri u32[N]; done u8[N]; nout u32[N]; elemrow u32[N+1]; elems u32[3 n_elems]
#pragma once

#include "common.cuh"
#include "lbvh.cuh"
#include "scan.cuh"

namespace sb {

constexpr uint32_t kLocal2 = 128;     // local ids per star (3 super nodes + inserted points)
constexpr uint32_t kMortonSeed = 8;   // Morton neighbours on each side inserted by insert_morton_neighbors
constexpr uint32_t kSuper2 = 3;       // super nodes (mesh.cpp:96-105)

struct Mesh2D {
    uint32_t n_nodes = 0, n_elems = 0;
    cudaStream_t stream = nullptr;
    DeviceBuffer<float4> nodes;  // input (x, y, 0, 0)
    LBVH3D lbvh;                 // bits = 64: the 2D Morton code of the points
    DeviceBuffer<uint32_t> loc, tri, nloc, ntri, nout, elemrow, elems;
    DeviceBuffer<uint8_t> done;
    DeviceBuffer<uint32_t> words;  // [0] status bits [1] incomplete stars after the last sweep
    DeviceBuffer<float> staging;
    DeviceBuffer<uint32_t> input_bad;  // set when the staged input holds an infinite or NaN value
    ScanPlan scan;
    PinnedWords pinned;
    uint32_t last_status = 0, last_incomplete = 0;
    bool inited = false, drop_super = false, compressed = false;

    Mesh2D();
    ~Mesh2D();
    // Host coordinates, nnodes x 2 row-major (mesh.cpp:818-823).
    void set_nodes_host(uint32_t n, const float* coords);
    void init();
    void insert_morton_neighbors();
    void insert_bvh_neighbors();
    void insert_iterative();
    void remove_super_nodes();
    // Owner-compressed triangles (mesh.cpp:664-697); returns their number.
    uint32_t compress();
    void read_status();
};

}  // namespace sb
