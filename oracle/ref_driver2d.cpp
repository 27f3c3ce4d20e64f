// Oracle driver over the reference's own 2D alpha shape (test infrastructure
// only).  A translation unit of its own: the reference's 3D header declares
// AlphaShape2D_set_nodes with an AlphaShape3D argument
// (include/mesh/DirectAlphaShape3D.hpp:52), so the two headers cannot meet.
//   * AlphaShape2D::{set_nodes, init, compute, compress}   (src/mesh/DirectAlphaShape2D.cpp:68-690)
//   * its LBVH<Sphere2D, InternalNodeDataFunctor, 2>        (include/mesh/DirectAlphaShape2D.hpp:84-98)
#include <cstdint>
#include <cstring>

#include "DirectAlphaShape2D.hpp"

using stream::mesh::AlphaShape2D;

extern "C" {

// Full run through the reference's C++ API; release with ref_ashape2d_free.
void* ref_ashape2d_run(uint32_t n, const float* coords, const float* alpha) {
    auto* a = new AlphaShape2D;
    auto h = AvaHostArray<Sphere2D, int>::create({(int)n});
    for (uint32_t i = 0; i < n; ++i) h(i) = {.c = Vec2f({coords[2 * i], coords[2 * i + 1]}), .r = alpha[i]};
    a->set_nodes(h);
    a->init();
    a->compute();
    a->compress();
    return a;
}

void ref_ashape2d_sizes(void* hnd, uint32_t* n_nodes, uint32_t* n_elems, uint32_t* n_edges) {
    auto* a = static_cast<AlphaShape2D*>(hnd);
    *n_nodes = a->n_nodes;
    *n_elems = a->n_elems;
    *n_edges = a->n_edges;
}

// perm[n], elems[n_elems x 3], row[n+1], neig[n_edges], edge_is_bnd[n_edges],
// node_is_bnd[n], nineig[n] (neighbours incl. the 3 infinity ids), nelem[n]
// (kept local triangles), coords_m[(n+3) x 3] (Morton-ordered x, y, alpha and
// the 3 infinity points).  Any pointer may be null.
void ref_ashape2d_get(void* hnd, uint32_t* perm, uint32_t* elems, uint32_t* row, uint32_t* neig,
                      uint8_t* edge_is_bnd, uint8_t* node_is_bnd, uint32_t* nineig, uint8_t* nelem,
                      float* coords_m) {
    auto* a = static_cast<AlphaShape2D*>(hnd);
    const uint32_t n = a->n_nodes;
    if (perm) std::memcpy(perm, a->lbvh.d_map_sorted->data, n * 4);
    if (elems) std::memcpy(elems, a->d_elemglob->data, (size_t)a->n_elems * 12);
    if (row) std::memcpy(row, a->d_row->data, (size_t)(n + 1) * 4);
    if (neig) std::memcpy(neig, a->d_neig->data, (size_t)a->n_edges * 4);
    if (edge_is_bnd) std::memcpy(edge_is_bnd, a->d_edge_is_bnd->data, a->n_edges);
    if (node_is_bnd) std::memcpy(node_is_bnd, a->d_node_is_bnd->data, n);
    if (nineig) std::memcpy(nineig, a->d_node_nineig->data, (size_t)n * 4);
    if (nelem) std::memcpy(nelem, a->d_node_nelem->data, n);
    if (coords_m) std::memcpy(coords_m, a->lbvh.d_obj_m->data, (size_t)(n + 3) * 12);
}

// The LBVH arrays: bb_glob[4] = pmin, pmax; morton_sorted[n]; sep[n-1];
// cil[n-1]; bboxes[(n-1) x 4] (min x, min y, max x, max y).  Any may be null.
void ref_ashape2d_lbvh(void* hnd, float* bb_glob, uint64_t* morton_sorted, int32_t* sep, uint8_t* cil,
                       float* bboxes) {
    auto* a = static_cast<AlphaShape2D*>(hnd);
    const uint32_t n = a->n_nodes;
    if (bb_glob) std::memcpy(bb_glob, a->lbvh.d_bb_glob->data, 4 * sizeof(float));
    if (morton_sorted) std::memcpy(morton_sorted, a->lbvh.d_morton_sorted->data, (size_t)n * 8);
    if (sep) std::memcpy(sep, a->lbvh.d_internal_sep->data, (size_t)(n - 1) * 4);
    if (cil) std::memcpy(cil, a->lbvh.d_child_is_leaf->data, n - 1);
    if (bboxes) std::memcpy(bboxes, a->lbvh.d_internal_data->data, (size_t)(n - 1) * 16);
}

// Neighbour lists in traversal order: out is n x width, UINT32_MAX padded (the
// first nineig[i] - 3 entries of row i are meaningful, at most 249).
void ref_ashape2d_candidates(void* hnd, uint32_t width, uint32_t* out) {
    auto* a = static_cast<AlphaShape2D*>(hnd);
    const uint32_t n = a->n_nodes;
    const auto tri = a->get_triloc_struct();
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t off = tri.d_block_offset_v(i / 32) + i % 32;
        const uint32_t k = a->d_node_nineig->data[i];
        for (uint32_t j = 0; j < width; ++j) {
            uint32_t v = 0xFFFFFFFFu;
            if (j + 3 < k) v = a->d_node_neig->data[off + j * 32];
            out[(size_t)i * width + j] = v;
        }
    }
}

void ref_ashape2d_free(void* hnd) { delete static_cast<AlphaShape2D*>(hnd); }

}  // extern "C"
