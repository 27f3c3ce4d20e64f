// extern "C" boundary of the 2D Delaunay mesher.  Entry points keep the
// reference's names and argument meaning (src/mesh/mesh.cpp:806-862);
// additive entry points return an int status (0 = ok).  No C++ exception
// crosses this boundary: reference-named void functions record failures in
// the handle (Mesh2D_get_status).
#include <vector>

#include "capi_common.cuh"
#include "mesh2d.cuh"
#include "stream_b200.h"

struct Mesh2D : sb::Mesh2D {};

namespace {
// Runs f and records a failure's status bits in the handle.
template <typename F>
void record(Mesh2D* m, F&& f) {
    m->last_status |= (uint32_t)sb_guard(f);
}
}  // namespace

extern "C" {

SB_EXPORT Mesh2D* Mesh2D_create(void) {
    Mesh2D* m = nullptr;
    sb_guard([&] { m = new Mesh2D; });
    return m;
}

SB_EXPORT void Mesh2D_destroy(Mesh2D* m) {
    sb_guard([&] { delete m; });
}

SB_EXPORT void Mesh2D_set_nodes(Mesh2D* m, uint32_t nnodes, const float* nodes) {
    if (!m) return;
    m->last_status = 0;  // a new point set: earlier failures no longer apply
    if (!nodes) {
        m->last_status |= sb::ST_BAD_INPUT;
        return;
    }
    record(m, [&] { m->set_nodes_host(nnodes, nodes); });
}

SB_EXPORT void Mesh2D_init(Mesh2D* m) {
    if (!m) return;
    record(m, [&] { m->init(); SB_CUDA(cudaStreamSynchronize(m->stream)); });
}

SB_EXPORT void Mesh2D_insert_morton_neighbors(Mesh2D* m) {
    if (!m) return;
    record(m, [&] { m->insert_morton_neighbors(); m->read_status(); });
}

SB_EXPORT void Mesh2D_insert_BVH_neighbors(Mesh2D* m) {
    if (!m) return;
    record(m, [&] { m->insert_bvh_neighbors(); m->read_status(); });
}

SB_EXPORT void Mesh2D_insert_iterative(Mesh2D* m) {
    if (!m) return;
    record(m, [&] {
        m->insert_iterative();
        m->read_status();
        if (m->last_incomplete) m->last_status |= sb::ST_INCOMPLETE;
    });
}

SB_EXPORT void Mesh2D_remove_super_nodes(Mesh2D* m) {
    if (!m) return;
    m->remove_super_nodes();
}

SB_EXPORT uint32_t Mesh2D_get_nelem(Mesh2D* m) {
    if (!m || !m->inited) return 0u;
    uint32_t ne = 0;
    record(m, [&] { ne = m->compress(); });
    return ne;
}

SB_EXPORT void Mesh2D_get_elem(Mesh2D* m, uint32_t* elems) {
    if (!m || !elems || !m->compressed) return;
    record(m, [&] {
        SB_CUDA(cudaMemcpyAsync(elems, m->elems.ptr, sizeof(uint32_t) * 3 * (size_t)m->n_elems, cudaMemcpyDeviceToHost,
                                m->stream));
        SB_CUDA(cudaStreamSynchronize(m->stream));
    });
}

SB_EXPORT void Mesh2D_get_ordered_nodes(Mesh2D* m, float* nodes) {
    if (!m || !nodes || !m->inited) return;
    record(m, [&] {
        std::vector<float4> h(m->n_nodes);
        SB_CUDA(cudaMemcpyAsync(h.data(), m->lbvh.obj_m.ptr, sizeof(float4) * m->n_nodes, cudaMemcpyDeviceToHost,
                                m->stream));
        SB_CUDA(cudaStreamSynchronize(m->stream));
        for (uint32_t i = 0; i < m->n_nodes; ++i) {
            nodes[2 * (size_t)i] = h[i].x;
            nodes[2 * (size_t)i + 1] = h[i].y;
        }
    });
}

// ---- additive entry points -------------------------------------------------
SB_EXPORT int Mesh2D_get_status(const Mesh2D* m) { return m ? (int)m->last_status : (int)sb::ST_BAD_INPUT; }

SB_EXPORT int Mesh2D_get_counters(const Mesh2D* m, uint32_t* out2) {
    if (!m || !out2) return (int)sb::ST_BAD_INPUT;
    out2[0] = m->last_status;
    out2[1] = m->last_incomplete;
    return 0;
}

SB_EXPORT uint32_t Mesh2D_get_permutation(const Mesh2D* m, uint32_t* perm) {
    if (!m || !perm || !m->inited) return 0u;
    const int rc = sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(perm, m->lbvh.perm.ptr, sizeof(uint32_t) * m->n_nodes, cudaMemcpyDeviceToHost,
                                m->stream));
        SB_CUDA(cudaStreamSynchronize(m->stream));
    });
    return rc ? 0u : m->n_nodes;
}

// The three super nodes (x, y pairs), as placed by init.
SB_EXPORT int Mesh2D_get_super_nodes(const Mesh2D* m, float* xy6) {
    if (!m || !xy6 || !m->inited) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        float4 h[3];
        SB_CUDA(cudaMemcpyAsync(h, m->lbvh.obj_m.ptr + m->n_nodes, sizeof h, cudaMemcpyDeviceToHost, m->stream));
        SB_CUDA(cudaStreamSynchronize(m->stream));
        for (int k = 0; k < 3; ++k) {
            xy6[2 * k] = h[k].x;
            xy6[2 * k + 1] = h[k].y;
        }
    });
}

}  // extern "C"
