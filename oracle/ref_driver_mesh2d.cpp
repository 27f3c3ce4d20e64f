// Oracle driver over the reference's Mesh2D (test infrastructure only), init
// stage only: the Morton order and the super nodes that Mesh2D_init
// (src/mesh/mesh.cpp:68-135) produces.  Its insertion phases push into a
// fixed-size traversal heap without a bound (mesh.cpp:471, 509, 548) and are
// not called.  A translation unit of its own (mesh.hpp and the alpha-shape
// headers declare overlapping names).
#include <cstdint>
#include <cstring>

#include "mesh.hpp"

extern "C" {

// perm[n]: ordered node i is input node perm[i]; coords_m[(n + 3) x 2]: the
// ordered nodes followed by the three super nodes.
void ref_mesh2d_order(uint32_t n, const float* xy, uint32_t* perm, float* coords_m) {
    Mesh2D* m = Mesh2D_create();
    Mesh2D_set_nodes(m, n, xy);
    Mesh2D_init(m);
    std::memcpy(perm, m->lbvh.d_map_sorted->data, (size_t)n * 4);
    std::memcpy(coords_m, m->lbvh.d_obj_m->data, (size_t)(n + 3) * 8);
    Mesh2D_destroy(m);
}

}  // extern "C"
