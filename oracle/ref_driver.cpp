// Oracle driver over the reference's own C++ API (test infrastructure only).
//
// Built by oracle/Makefile together with the reference's unmodified sources
// (compiled for the host against oracle/ava_shim) into oracle/_ref/libstream_ref.so.
// It exposes flat extern "C" entry points that dump the reference's
// intermediate and final arrays so tests can compare them with the CUDA path:
//   * LBVH<Sphere3D, ComputeBB_Functor<Sphere3D>, 3>::build   (include/geometry/lbvh.hpp:354-360)
//   * AlphaShape3D::{set_nodes, init, compute, compress}    (src/mesh/DirectAlphaShape3D.cpp:68-743)
//   * ConjugateGradient::{solve_precond, solve}              (src/numerics/conjugate_gradient.cpp:61-208)
// The reference's own C ABI (AlphaShape3D_*, d_csr_*, ...) is exported by the
// same library, since its sources are compiled in unmodified.
#include <cstdint>
#include <cstring>
#include <vector>

#include "DirectAlphaShape3D.hpp"
#include "lbvh.hpp"
#include "lbvh_agglo.hpp"
#include "trbvh.hpp"
#include "csr.hpp"
#include "linear_system.hpp"
#include "preconditioner.hpp"
#include "solver.hpp"

using stream::mesh::AlphaShape3D;

extern "C" {

// LBVH over 3D spheres.  xyzr: n x 4 floats (x, y, z, r).  Outputs (may be null):
// bb_glob[6] = pmin, pmax; morton_sorted[n]; perm[n]; sep[n-1]; cil[n-1];
// leaf_parent[n]; internal_parent[n-1]; bboxes[(n-1) x 6]; obj_m[n x 4].
int ref_lbvh3d(uint32_t n, const float* xyzr, float* bb_glob, uint64_t* morton_sorted,
               uint32_t* perm, int32_t* sep, uint8_t* cil, uint32_t* leaf_parent,
               uint32_t* internal_parent, float* bboxes, float* obj_m) {
    if (n < 2) return 1;
    auto h = AvaHostArray<Sphere3D, int>::create({(int)n});
    for (uint32_t i = 0; i < n; ++i)
        h(i) = {.c = Vec3f({xyzr[4 * i], xyzr[4 * i + 1], xyzr[4 * i + 2]}), .r = xyzr[4 * i + 3]};
    auto d = AvaDeviceArray<Sphere3D, int>::create({(int)n});
    d->set(h);
    Sphere3DLBVH lbvh;
    lbvh.set_objects(d);
    lbvh.build();
    if (bb_glob) std::memcpy(bb_glob, lbvh.d_bb_glob->data, 6 * sizeof(float));
    if (morton_sorted) std::memcpy(morton_sorted, lbvh.d_morton_sorted->data, n * 8);
    if (perm) std::memcpy(perm, lbvh.d_map_sorted->data, n * 4);
    if (sep) std::memcpy(sep, lbvh.d_internal_sep->data, (n - 1) * 4);
    if (cil) std::memcpy(cil, lbvh.d_child_is_leaf->data, (n - 1));
    if (leaf_parent) std::memcpy(leaf_parent, lbvh.d_leaf_parent->data, n * 4);
    if (internal_parent) std::memcpy(internal_parent, lbvh.d_internal_parent->data, (n - 1) * 4);
    if (bboxes) std::memcpy(bboxes, lbvh.d_internal_data->data, (size_t)(n - 1) * 24);
    if (obj_m) std::memcpy(obj_m, lbvh.d_obj_m->data, (size_t)n * 16);
    return 0;
}

// TRBVH over 3D spheres (include/geometry/trbvh.hpp).  optimize = 0 stops
// after the Apetrei build (_build_hierarchy, :299-390); 1 runs build() with its
// three treelet_optimize rounds (:637-679).  Node ids: leaves 0..n-1, internal
// nodes n..2n-2.  Outputs (may be null): child_left/right[n-1],
// range_min/max[n-1], parent[2n-1], bboxes[(2n-1) x 6], subtree_size[2n-1],
// sah[2n-1], root[1], obj_m[n x 4].
int ref_trbvh3d(uint32_t n, const float* xyzr, int optimize, uint32_t* child_left, uint32_t* child_right,
                uint32_t* range_min, uint32_t* range_max, uint32_t* parent, float* bboxes,
                uint32_t* subtree_size, float* sah, uint32_t* root, float* obj_m) {
    if (n < 2) return 1;
    auto h = AvaHostArray<Sphere3D, int>::create({(int)n});
    for (uint32_t i = 0; i < n; ++i)
        h(i) = {.c = Vec3f({xyzr[4 * i], xyzr[4 * i + 1], xyzr[4 * i + 2]}), .r = xyzr[4 * i + 3]};
    auto d = AvaDeviceArray<Sphere3D, int>::create({(int)n});
    d->set(h);
    Sphere3DTRBVH t;
    t.set_objects(d);
    if (optimize) {
        t.build();
    } else {
        t._compute_global_bbox();
        t._compute_morton_codes();
        t._sort_objects();
        t._build_hierarchy();
    }
    const size_t m = 2 * (size_t)n - 1;
    if (child_left) std::memcpy(child_left, t.d_child_left->data, (n - 1) * 4);
    if (child_right) std::memcpy(child_right, t.d_child_right->data, (n - 1) * 4);
    if (range_min) std::memcpy(range_min, t.d_range_min->data, (n - 1) * 4);
    if (range_max) std::memcpy(range_max, t.d_range_max->data, (n - 1) * 4);
    if (parent) std::memcpy(parent, t.d_parent->data, m * 4);
    if (bboxes) std::memcpy(bboxes, t.d_bboxes->data, m * 24);
    if (subtree_size) std::memcpy(subtree_size, t.d_subtree_size->data, m * 4);
    if (sah) std::memcpy(sah, t.d_sah_cost->data, m * 4);
    if (root) std::memcpy(root, t.d_root->data, 4);
    if (obj_m) std::memcpy(obj_m, t.d_obj_m->data, (size_t)n * 16);
    return 0;
}

// LBVHa over 3D spheres (include/geometry/lbvh_agglo.hpp: Apetrei's
// agglomerative build, :270-325), the build() stages without the timing
// prints.  children[n-1][2], range[n-1][2], parent[2n-1] (leaves 0..n-1,
// internal nodes n..2n-2, root parent 2n), boxes[2n-1] (6 floats), root[1],
// obj_m[n x 4].
int ref_lbvha3d(uint32_t n, const float* xyzr, uint32_t* children, uint32_t* range, uint32_t* parent,
                float* boxes, uint32_t* root, float* obj_m) {
    if (n < 2) return 1;
    auto h = AvaHostArray<Sphere3D, int>::create({(int)n});
    for (uint32_t i = 0; i < n; ++i)
        h(i) = {.c = Vec3f({xyzr[4 * i], xyzr[4 * i + 1], xyzr[4 * i + 2]}), .r = xyzr[4 * i + 3]};
    auto d = AvaDeviceArray<Sphere3D, int>::create({(int)n});
    d->set(h);
    stream::geo::LBVHa<Sphere3D, stream::geo::ComputeBB_Functor<Sphere3D>, 3> t;
    t.set_objects(d);
    t._compute_global_bbox();
    t._compute_morton_codes();
    t._sort_objects();
    t._build_hierarchy();
    const size_t m = 2 * (size_t)n - 1;
    if (children) std::memcpy(children, t.d_children->data, (n - 1) * 8);
    if (range) std::memcpy(range, t.d_range->data, (n - 1) * 8);
    if (parent) std::memcpy(parent, t.d_parent->data, m * 4);
    if (boxes) std::memcpy(boxes, t.d_internal_data->data, m * 24);
    if (root) std::memcpy(root, t.d_root->data, 4);
    if (obj_m) std::memcpy(obj_m, t.d_obj_m->data, (size_t)n * 16);
    return 0;
}

// Full alpha-shape run through the reference's C++ API.  Returns an opaque
// handle; query with ref_ashape3d_sizes / ref_ashape3d_get, release with
// ref_ashape3d_free.
void* ref_ashape3d_run(uint32_t n, const float* coords, const float* alpha) {
    auto* a = new AlphaShape3D;
    auto h = AvaHostArray<Sphere3D, int>::create({(int)n});
    for (uint32_t i = 0; i < n; ++i)
        h(i) = {.c = Vec3f({coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]}), .r = alpha[i]};
    a->set_nodes(h);
    a->init();
    a->compute();
    a->compress();
    return a;
}

void ref_ashape3d_sizes(void* hnd, uint32_t* n_nodes, uint32_t* n_elems, uint32_t* n_edges) {
    auto* a = static_cast<AlphaShape3D*>(hnd);
    *n_nodes = a->n_nodes;
    *n_elems = a->n_elems;
    *n_edges = a->n_edges;
}

// perm[n], elems[n_elems x 4], row[n+1], neig[n_edges], edge_is_bnd[n_edges],
// node_is_bnd[n], nineig[n] (neighbours incl. the 4 infinity ids, capped at 128),
// nelem[n] (kept local tets), coords_m[(n+4) x 4] (Morton-ordered spheres and
// the 4 infinity points).  Any pointer may be null.
void ref_ashape3d_get(void* hnd, uint32_t* perm, uint32_t* elems, uint32_t* row, uint32_t* neig,
                      uint8_t* edge_is_bnd, uint8_t* node_is_bnd, uint32_t* nineig,
                      uint8_t* nelem, float* coords_m) {
    auto* a = static_cast<AlphaShape3D*>(hnd);
    const uint32_t n = a->n_nodes;
    if (perm) std::memcpy(perm, a->lbvh.d_map_sorted->data, n * 4);
    if (elems) std::memcpy(elems, a->d_elemglob->data, (size_t)a->n_elems * 16);
    if (row) std::memcpy(row, a->d_row->data, (size_t)(n + 1) * 4);
    if (neig) std::memcpy(neig, a->d_neig->data, (size_t)a->n_edges * 4);
    if (edge_is_bnd) std::memcpy(edge_is_bnd, a->d_edge_is_bnd->data, a->n_edges);
    if (node_is_bnd) std::memcpy(node_is_bnd, a->d_node_is_bnd->data, n);
    if (nineig) std::memcpy(nineig, a->d_node_nineig->data, (size_t)n * 4);
    if (nelem) std::memcpy(nelem, a->d_node_nelem->data, n);
    if (coords_m) std::memcpy(coords_m, a->lbvh.d_obj_m->data, (size_t)(n + 4) * 16);
}

// Candidate neighbour lists in traversal order (first nineig[i]-4 entries of
// each row are meaningful; max 124 per row).  out: n x 124, UINT32_MAX padded.
void ref_ashape3d_candidates(void* hnd, uint32_t* out) {
    auto* a = static_cast<AlphaShape3D*>(hnd);
    const uint32_t n = a->n_nodes;
    const auto tri = a->get_triloc_struct();
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t off = tri.d_block_offset_v(i / 32) + i % 32;
        const uint32_t k = a->d_node_nineig->data[i];
        for (uint32_t j = 0; j < 124; ++j) {
            uint32_t v = 0xFFFFFFFFu;
            if (j + 4 < k) v = a->d_node_neig->data[off + j * 32];
            out[(size_t)i * 124 + j] = v;
        }
    }
}

void ref_ashape3d_free(void* hnd) { delete static_cast<AlphaShape3D*>(hnd); }

// Reference FP32 CG / Jacobi-PCG on a host CSR.  x is in/out.  Returns the
// iteration counter exactly as the reference computes it.
uint32_t ref_cg_solve(uint32_t n, const uint32_t* row, const uint32_t* col, const float* val,
                      const float* b, float* x, int jacobi) {
    h_CSR* hc = h_csr_create(n, row, col, val);
    d_CSR* dc = d_csr_create();
    d_csr_h2d(dc, hc);
    LinSys* sys = LinSys_create();
    LinSys_set(sys, dc, b);
    SolverCG* cg = SolverCG_create();
    uint32_t it;
    if (jacobi) {
        PrecJacobi_st* p = PrecJacobi_create(dc);
        it = SolverCG_jacobi_solve(cg, sys, p, x);
        PrecJacobi_destroy(p);
    } else {
        it = SolverCG_solve(cg, sys, x);
    }
    SolverCG_destroy(cg);
    LinSys_destroy(sys);
    d_csr_destroy(dc);
    h_csr_destroy(hc);
    return it;
}

}  // extern "C"
