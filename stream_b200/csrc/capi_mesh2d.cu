// extern "C" boundary of the 2D mesher.  Entry points keep the reference's
// names and argument meaning (src/mesh/DirectAlphaShape2D.cpp:698-753);
// additive entry points return an int status (0 = ok).  No C++ exception
// crosses this boundary.
#include <algorithm>
#include <vector>

#include "ashape2d.cuh"
#include "capi_common.cuh"
#include "stream_b200.h"

struct AlphaShape2D : sb::AlphaShape2D {};

extern "C" {

SB_EXPORT AlphaShape2D* AlphaShape2D_create(void) {
    AlphaShape2D* a = nullptr;
    sb_guard([&] { a = new AlphaShape2D; });
    return a;
}

SB_EXPORT void AlphaShape2D_destroy(AlphaShape2D* a) {
    sb_guard([&] { delete a; });
}

SB_EXPORT void AlphaShape2D_set_nodes(AlphaShape2D* a, uint32_t nnodes, const float* coords, const float* alpha) {
    if (!a) return;
    a->last_status = 0;  // a new point set: earlier failures no longer apply
    if (!coords || !alpha || sb_guard([&] { a->set_nodes_host(nnodes, coords, alpha); }))
        a->last_status |= sb::ST_BAD_INPUT;
}

SB_EXPORT void AlphaShape2D_init(AlphaShape2D* a) {
    if (!a) return;
    if (sb_guard([&] { a->init(); SB_CUDA(cudaStreamSynchronize(a->stream)); })) a->last_status |= sb::ST_CUDA_ERROR;
}

SB_EXPORT void AlphaShape2D_compute(AlphaShape2D* a) {
    if (!a) return;
    if (sb_guard([&] { a->compute(); a->read_counters(); })) a->last_status |= sb::ST_CUDA_ERROR;
}

SB_EXPORT uint32_t AlphaShape2D_get_nelem(const AlphaShape2D* a) { return a ? a->n_elems : 0u; }

SB_EXPORT void AlphaShape2D_get_elem(const AlphaShape2D* a, uint32_t* elems) {
    if (!a || !elems || !a->computed) return;
    sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(elems, a->elems.ptr, sizeof(uint32_t) * 3 * (size_t)a->n_elems,
                                cudaMemcpyDeviceToHost, a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
}

SB_EXPORT void AlphaShape2D_get_ordered_nodes(AlphaShape2D* a, float* nodes) {
    if (!a || !nodes || !a->inited) return;
    sb_guard([&] {
        std::vector<float4> h(a->n_nodes);
        SB_CUDA(cudaMemcpyAsync(h.data(), a->lbvh.obj_m.ptr, sizeof(float4) * a->n_nodes, cudaMemcpyDeviceToHost,
                                a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
        for (uint32_t i = 0; i < a->n_nodes; ++i) {
            nodes[2 * (size_t)i] = h[i].x;
            nodes[2 * (size_t)i + 1] = h[i].y;
        }
    });
}

// ---- additive entry points -------------------------------------------------
SB_EXPORT int AlphaShape2D_set_nodes_device(AlphaShape2D* a, uint32_t nnodes, const float* d_xy0a) {
    if (!a || !d_xy0a || nnodes < 2) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] { a->set_nodes_device(nnodes, reinterpret_cast<const float4*>(d_xy0a)); });
}

SB_EXPORT int AlphaShape2D_get_status(const AlphaShape2D* a) { return a ? (int)a->last_status : (int)sb::ST_BAD_INPUT; }

SB_EXPORT int AlphaShape2D_get_counters(const AlphaShape2D* a, uint32_t* out3) {
    if (!a || !out3) return (int)sb::ST_BAD_INPUT;
    out3[0] = a->last_status;
    out3[1] = a->last_limited;
    out3[2] = a->last_exact;
    return 0;
}

SB_EXPORT uint32_t AlphaShape2D_get_permutation(const AlphaShape2D* a, uint32_t* perm) {
    if (!a || !perm || !a->inited) return 0u;
    const int rc = sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(perm, a->lbvh.perm.ptr, sizeof(uint32_t) * a->n_nodes, cudaMemcpyDeviceToHost,
                                a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
    return rc ? 0u : a->n_nodes;
}

SB_EXPORT uint32_t AlphaShape2D_get_nedge(const AlphaShape2D* a) { return a ? a->n_edges : 0u; }

SB_EXPORT uint32_t AlphaShape2D_get_edges(const AlphaShape2D* a, uint32_t* row, uint32_t* neig, uint8_t* edge_is_bnd) {
    if (!a || !a->computed) return 0u;
    const int rc = sb_guard([&] {
        if (row)
            SB_CUDA(cudaMemcpyAsync(row, a->row.ptr, sizeof(uint32_t) * ((size_t)a->n_nodes + 1),
                                    cudaMemcpyDeviceToHost, a->stream));
        if (neig)
            SB_CUDA(cudaMemcpyAsync(neig, a->neig.ptr, sizeof(uint32_t) * a->n_edges, cudaMemcpyDeviceToHost, a->stream));
        if (edge_is_bnd)
            SB_CUDA(cudaMemcpyAsync(edge_is_bnd, a->edge_is_bnd.ptr, a->n_edges, cudaMemcpyDeviceToHost, a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
    return rc ? 0u : a->n_edges;
}

SB_EXPORT uint32_t AlphaShape2D_get_boundary_nodes(const AlphaShape2D* a, uint8_t* is_bnd) {
    if (!a || !is_bnd || !a->computed) return 0u;
    const int rc = sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(is_bnd, a->node_is_bnd.ptr, a->n_nodes, cudaMemcpyDeviceToHost, a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
    return rc ? 0u : a->n_nodes;
}

// Per-star diagnostics in Morton order: nineig (star size incl. the 3
// infinity ids), nkeep (kept local triangles), neighbour rows (n x width,
// traversal order, UINT32_MAX past nineig - 3).  Any pointer may be null.
SB_EXPORT int AlphaShape2D_get_stars(const AlphaShape2D* a, uint32_t* nineig, uint8_t* nkeep, uint32_t* cand,
                                     uint32_t width) {
    if (!a || !a->computed) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const uint32_t n = a->n_nodes;
        std::vector<uint32_t> k(n);
        SB_CUDA(cudaMemcpyAsync(k.data(), a->nineig.ptr, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, a->stream));
        if (nkeep) SB_CUDA(cudaMemcpyAsync(nkeep, a->nkeep.ptr, n, cudaMemcpyDeviceToHost, a->stream));
        std::vector<uint32_t> ell, boff;
        if (cand) {
            const uint32_t W = (n + 31) / 32;
            boff.resize((size_t)W + 1);
            ell.resize(a->slots);
            SB_CUDA(cudaMemcpyAsync(boff.data(), a->boff.ptr, sizeof(uint32_t) * boff.size(), cudaMemcpyDeviceToHost,
                                    a->stream));
            if (a->slots)
                SB_CUDA(cudaMemcpyAsync(ell.data(), a->cand.ptr, sizeof(uint32_t) * a->slots, cudaMemcpyDeviceToHost,
                                        a->stream));
        }
        SB_CUDA(cudaStreamSynchronize(a->stream));
        if (nineig) std::copy(k.begin(), k.end(), nineig);
        if (cand)
            for (uint32_t i = 0; i < n; ++i)
                for (uint32_t j = 0; j < width; ++j)
                    cand[(size_t)i * width + j] =
                        j + sb::kInf2 < k[i] ? ell[(size_t)boff[i >> 5] + 32 * (size_t)(j + sb::kInf2) + (i & 31)] : 0xFFFFFFFFu;
    });
}

SB_EXPORT int AlphaShape2D_set_profiling(AlphaShape2D* a, int on) {
    if (!a) return (int)sb::ST_BAD_INPUT;
    a->profiling = on != 0;
    return 0;
}

// ms6 = {LBVH build + infinity points, count pass + ELL layout, fill pass,
// star, scans + size read-back, compress} of the last init()+compute().
SB_EXPORT int AlphaShape2D_get_profile(AlphaShape2D* a, float* ms6) {
    if (!a || !ms6 || !a->profiling || !a->computed) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        a->collect_profile();
        static_assert(sb::AlphaShape2D::S_COUNT == 6, "ms6 holds one value per stage");
        for (int i = 0; i < sb::AlphaShape2D::S_COUNT; ++i) ms6[i] = a->stage_ms[i];
    });
}

SB_EXPORT int AlphaShape2D_set_stream(AlphaShape2D* a, void* stream) {
    if (!a) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] { a->set_stream(static_cast<cudaStream_t>(stream)); });
}

SB_EXPORT int AlphaShape2D_synchronize(AlphaShape2D* a) {
    if (!a) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] { SB_CUDA(cudaStreamSynchronize(a->stream)); });
}

}  // extern "C"
