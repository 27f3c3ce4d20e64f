// Oracle (test infrastructure only): plain-C restatement of the reference's
// PFEM remesh-and-solve path.  Nothing in the product links this; tests,
// __graft_entry__.smoke() and bench.py's CPU baseline load it through ctypes
// as the checker.  Each function cites the reference file:line it restates.
#ifndef STREAM_ORACLE_H
#define STREAM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// ---- predicates (orc_predicates.c; include/geometry/predicates.hpp) -------
float orc_orient3d_exact(const float* pa, const float* pb, const float* pc, const float* pd);
float orc_orient3d(const float* pa, const float* pb, const float* pc, const float* pd);
float orc_insphere_exact(const float* pa, const float* pb, const float* pc, const float* pd,
                         const float* pe);
float orc_insphere_filter(const float* pa, const float* pb, const float* pc, const float* pd,
                          const float* pe, float* err);
float orc_conflict_det(const float* const pts[5], const uint32_t ids[5], int* used_exact);
// Batched form for tests: pts is m x 5 x 3 floats, ids m x 5; out m dets.
void orc_conflict_batch(uint32_t m, const float* pts, const uint32_t* ids, float* out,
                        uint8_t* used_exact);

// ---- LBVH (orc_lbvh.c; include/geometry/lbvh.hpp) -------------------------
// Global AABB of spheres xyzr (n x 4), inflated by each radius (fit_point=0)
// or of the centres only (fit_point=1).  out: pmin[3], pmax[3].
void orc_bbox3d(uint32_t n, const float* xyzr, int use_radius, float out[6]);
// Morton codes of the centres.  bits = 63 (21 per axis, lbvh.hpp:185-212) or
// 30 (10 per axis, morton.hpp:47-59 with the same quantisation).
void orc_morton3d(uint32_t n, const float* xyzr, const float bb[6], int bits, uint64_t* codes);
// Stable ascending LSD radix sort of (key, value) pairs, in place.
void orc_sort_pairs(uint32_t n, uint64_t* keys, uint32_t* vals);
// Karras hierarchy over sorted codes (lbvh.hpp:246-308).
void orc_karras(uint32_t n, const uint64_t* codes, int32_t* sep, uint8_t* cil,
                uint32_t* leaf_parent, uint32_t* internal_parent);
// Bottom-up node boxes (lbvh.hpp:311-351).  fit_point=1 uses the centre
// (DirectAlphaShape3D.hpp:92-104), 0 the sphere box (primitives.hpp:136-141).
void orc_fit(uint32_t n, const float* obj_m, const int32_t* sep, const uint8_t* cil,
             int fit_point, float* bboxes);
// Full build: bb_glob[6], codes_sorted[n], perm[n], sep, cil, leaf_parent,
// internal_parent, bboxes[(n-1) x 6], obj_m[n x 4].  Any output may be null.
int orc_lbvh3d(uint32_t n, const float* xyzr, int bits, int fit_point, float* bb_glob,
               uint64_t* codes_sorted, uint32_t* perm, int32_t* sep, uint8_t* cil,
               uint32_t* leaf_parent, uint32_t* internal_parent, float* bboxes, float* obj_m);

// ---- TRBVH (orc_trbvh.c; include/geometry/trbvh.hpp) ----------------------
typedef struct {
    uint32_t n, root;
    uint32_t *child_left, *child_right;  // n-1 (internal node i = id n+i)
    uint32_t *range_min, *range_max;     // n-1 (Apetrei build ranges)
    uint32_t* parent;                    // 2n-1 (root parent = 2n)
    float* bboxes;                       // (2n-1) x 6
    uint32_t* subtree_size;              // 2n-1
    float* sah;                          // 2n-1 (order-independent SAH)
    float* obj_m;                        // n x 4
} orc_trbvh;
// rounds = 0: Apetrei build only; 3: the reference's three treelet rounds
// (min sizes K, 2K, 4K).  area3d: 0 = ext_x*ext_y (reference), 1 = xy+yz+zx.
int orc_trbvh3d(uint32_t n, const float* xyzr, int treelet_size, int area3d, int rounds, orc_trbvh* t);
void orc_trbvh3d_free(orc_trbvh* t);
void orc_trbvh3d_count(const orc_trbvh* t, uint32_t* out);

// ---- alpha shape (orc_ashape.c; src/mesh/DirectAlphaShape3D.cpp) ----------
#define ORC_STAR_CAP 128   // local ids per star incl. the 4 infinity points
typedef struct {
    uint32_t n, n_elems, n_edges;
    uint32_t status;        // bit flags, see ORC_ERR_*
    uint32_t n_truncated;   // stars with more candidates than the cap
    uint32_t n_exact;       // conflict tests that needed the exact path
    uint32_t* perm;         // n      Morton permutation (getPermutation)
    float* coords_m;        // (n+4) x 4  Morton-ordered spheres + 4 infinity points
    uint32_t* nineig;       // n      star size incl. infinity ids, capped
    uint32_t* cand;         // n x 124 candidate neighbours (global, traversal order)
    uint32_t* elemrow;      // n+1
    uint32_t* elems;        // n_elems x 4
    uint32_t* row;          // n+1
    uint32_t* neig;         // n_edges
    uint8_t* edge_is_bnd;   // n_edges
    uint8_t* node_is_bnd;   // n
    uint8_t* nelem;         // n      kept tets per star
} orc_ashape;
#define ORC_ERR_STACK 1u    // BVH traversal stack overflow
#define ORC_ERR_WALK 2u     // cavity boundary walk hit its 100-iteration cap
#define ORC_ERR_CYCLE 4u    // broken cavity boundary cycle
#define ORC_ERR_CAP 8u      // local tet list overflow
int orc_ashape3d(uint32_t n, const float* coords, const float* alpha, int bits, orc_ashape* out);
void orc_ashape3d_free(orc_ashape* a);

// ---- 2D (orc_predicates.c, orc_lbvh.c, orc_ashape2d.c) ---------------------
// include/geometry/predicates.hpp:337-589; lbvh.hpp with dim = 2;
// src/mesh/DirectAlphaShape2D.cpp.
float orc_orient2d_exact(const float* pa, const float* pb, const float* pc);
float orc_orient2d(const float* pa, const float* pb, const float* pc);
float orc_incircle_filter(const float* pa, const float* pb, const float* pc, const float* pd, float* err);
float orc_incircle_exact(const float* pa, const float* pb, const float* pc, const float* pd);
// s: n x 4 floats (x, y, unused, r); out/bb: pmin[2], pmax[2].
void orc_bbox2d(uint32_t n, const float* s, float out[4]);
void orc_morton2d(uint32_t n, const float* s, const float bb[4], uint64_t* codes);
typedef struct {
    uint32_t n, n_elems, n_edges;
    uint32_t status;        // ORC_ERR_* bits
    uint32_t n_exact;       // in-circle tests that needed the exact path
    float bb_glob[4];       // pmin, pmax (radius included)
    uint64_t* codes;        // n sorted Morton codes
    uint32_t* perm;         // n
    float* coords_m;        // (n+3) x 4  Morton-ordered (x, y, 0, alpha) + 3 infinity points
    uint32_t* nineig;       // n      neighbours incl. the 3 infinity ids (fill pass)
    uint32_t* row_offset;   // n+1    neighbour rows of the count pass
    uint32_t* cand;         // row_offset[n]  neighbours (global ids, traversal order)
    uint32_t* elemrow;      // n+1
    uint32_t* elems;        // n_elems x 3
    uint32_t* row;          // n+1
    uint32_t* neig;         // n_edges
    uint8_t* edge_is_bnd;   // n_edges
    uint8_t* node_is_bnd;   // n
    uint8_t* nelem;         // n      kept triangles per star
} orc_ashape2d_out;
int orc_ashape2d(uint32_t n, const float* coords, const float* alpha, orc_ashape2d_out* out);
void orc_ashape2d_free(orc_ashape2d_out* a);

// ---- solver (orc_cg.c; src/numerics/conjugate_gradient.cpp) ---------------
// FP32 CG / Jacobi-PCG with the reference's stopping rule and iteration count.
uint32_t orc_cg_f32(uint32_t n, const uint32_t* row, const uint32_t* col, const float* val,
                    const float* b, float* x, int jacobi);

#ifdef __cplusplus
}
#endif
#endif
