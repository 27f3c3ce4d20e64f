// extern "C" boundary for the mesher and the LBVH.  Entry points keep the
// reference's names and argument meaning (src/mesh/DirectAlphaShape3D.cpp:
// 754-810); additive entry points return an int status (0 = ok).  No C++
// exception crosses this boundary: failures are recorded in the handle's
// status word and in a thread-local message (stream_b200_last_error).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "capi_types.cuh"
#include "lbvh.cuh"
#include "trbvh.cuh"

// The opaque handle types of the C header are the library's classes
// (AlphaShape3D in capi_types.cuh).

namespace {
// CUDA events recorded between the stages of a tree build (profiling only).
struct BuildEvents {
    static constexpr int kMax = 8;
    cudaEvent_t ev[kMax] = {};
    int count = 0;
    bool on = false;
    cudaStream_t stream = nullptr;
    void begin(cudaStream_t s) {
        stream = s;
        count = 0;
        if (on) record();
    }
    void record() {
        if (!on || count >= kMax) return;
        if (!ev[count]) SB_CUDA(cudaEventCreate(&ev[count]));
        SB_CUDA(cudaEventRecord(ev[count], stream));
        ++count;
    }
    // Stage times (ms) between consecutive marks; returns the number written.
    uint32_t elapsed(float* ms, uint32_t cap) {
        if (!on || count < 2) return 0;
        SB_CUDA(cudaEventSynchronize(ev[count - 1]));
        uint32_t k = 0;
        for (int i = 0; i + 1 < count && k < cap; ++i, ++k) SB_CUDA(cudaEventElapsedTime(&ms[k], ev[i], ev[i + 1]));
        return k;
    }
    ~BuildEvents() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
};
}  // namespace

// Stages: global box + Morton codes + histograms, radix sort, gather, Karras
// hierarchy + fit.
struct Sphere3DLBVH : sb::LBVH3D::StageMarks {
    sb::LBVH3D bvh;
    sb::DeviceBuffer<float4> objs;
    sb::DeviceBuffer<uint32_t> status;
    cudaStream_t stream = nullptr;
    BuildEvents marks;
    Sphere3DLBVH() { SB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); status.ensure(1); }
    ~Sphere3DLBVH() { if (stream) cudaStreamDestroy(stream); }
    void mark_sort() override { marks.record(); }
    void mark_gather() override { marks.record(); }
    void mark_hierarchy() override { marks.record(); }
};

// Stages: global box + Morton codes + histograms, radix sort, gather, Apetrei
// build, treelet restructuring rounds.
struct Sphere3DTRBVH : sb::TRBVH3D::StageMarks {
    sb::TRBVH3D t;
    sb::DeviceBuffer<float4> objs;
    sb::DeviceBuffer<uint32_t> status, counts;
    cudaStream_t stream = nullptr;
    BuildEvents marks;
    Sphere3DTRBVH() { SB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); status.ensure(1); }
    ~Sphere3DTRBVH() { if (stream) cudaStreamDestroy(stream); }
    void mark_sort() override { marks.record(); }
    void mark_gather() override { marks.record(); }
    void mark_hierarchy() override { marks.record(); }
    void mark_treelets() override { marks.record(); }
};

extern "C" {

// ---------------------------------------------------------------- mesh ----
SB_EXPORT AlphaShape3D* AlphaShape3D_create(void) {
    AlphaShape3D* a = nullptr;
    sb_guard([&] { a = new AlphaShape3D; });
    return a;
}

SB_EXPORT void AlphaShape3D_destroy(AlphaShape3D* a) {
    sb_guard([&] { delete a; });
}

SB_EXPORT void AlphaShape3D_set_nodes(AlphaShape3D* a, uint32_t nnodes, const float* coords, const float* alpha) {
    if (!a) return;
    a->last_status = 0;  // a new point set: earlier failures no longer apply
    if (sb_guard([&] { a->set_nodes_host(nnodes, coords, alpha); })) a->last_status |= sb::ST_BAD_INPUT;
}

SB_EXPORT void AlphaShape3D_init(AlphaShape3D* a) {
    if (!a) return;
    if (sb_guard([&] { a->init(); SB_CUDA(cudaStreamSynchronize(a->stream)); })) a->last_status |= sb::ST_CUDA_ERROR;
}

SB_EXPORT void AlphaShape3D_compute(AlphaShape3D* a) {
    if (!a) return;
    if (sb_guard([&] { a->compute(); a->read_counters(); })) a->last_status |= sb::ST_CUDA_ERROR;
}

SB_EXPORT uint32_t AlphaShape3D_get_nelem(const AlphaShape3D* a) { return a ? a->n_elems : 0u; }

SB_EXPORT void AlphaShape3D_get_elem(const AlphaShape3D* a, uint32_t* elems) {
    if (!a || !elems || !a->computed) return;
    sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(elems, a->elems.ptr, sizeof(uint4) * (size_t)a->n_elems, cudaMemcpyDeviceToHost,
                                a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
}

SB_EXPORT void AlphaShape3D_get_ordered_nodes(AlphaShape3D* a, float* nodes) {
    if (!a || !nodes || !a->inited) return;
    sb_guard([&] {
        std::vector<float4> h(a->n_nodes);
        SB_CUDA(cudaMemcpyAsync(h.data(), a->lbvh.obj_m.ptr, sizeof(float4) * a->n_nodes, cudaMemcpyDeviceToHost,
                                a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
        for (uint32_t i = 0; i < a->n_nodes; ++i) {
            nodes[3 * (size_t)i] = h[i].x;
            nodes[3 * (size_t)i + 1] = h[i].y;
            nodes[3 * (size_t)i + 2] = h[i].z;
        }
    });
}

// ---- additive entry points -------------------------------------------------
SB_EXPORT int AlphaShape3D_set_morton_bits(AlphaShape3D* a, int bits) {
    if (!a || (bits != 63 && bits != 30)) return (int)sb::ST_BAD_INPUT;
    a->bits = bits;
    a->inited = a->computed = false;
    return 0;
}

SB_EXPORT int AlphaShape3D_set_nodes_device(AlphaShape3D* a, uint32_t nnodes, const float* d_xyza) {
    if (!a || !d_xyza || nnodes < 2) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] { a->set_nodes_device(nnodes, reinterpret_cast<const float4*>(d_xyza)); });
}

SB_EXPORT int AlphaShape3D_get_status(const AlphaShape3D* a) { return a ? (int)a->last_status : (int)sb::ST_BAD_INPUT; }

SB_EXPORT int AlphaShape3D_get_counters(const AlphaShape3D* a, uint32_t* out4) {
    if (!a || !out4) return (int)sb::ST_BAD_INPUT;
    out4[0] = a->last_status;
    out4[1] = a->last_deferred;
    out4[2] = a->last_truncated;
    out4[3] = a->last_exact;
    return 0;
}

SB_EXPORT uint32_t AlphaShape3D_get_permutation(const AlphaShape3D* a, uint32_t* perm) {
    if (!a || !perm || !a->inited) return 0u;
    const int rc = sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(perm, a->lbvh.perm.ptr, sizeof(uint32_t) * a->n_nodes, cudaMemcpyDeviceToHost,
                                a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
    return rc ? 0u : a->n_nodes;
}

SB_EXPORT uint32_t AlphaShape3D_get_nedge(const AlphaShape3D* a) { return a ? a->n_edges : 0u; }

SB_EXPORT uint32_t AlphaShape3D_get_edges(const AlphaShape3D* a, uint32_t* row, uint32_t* neig, uint8_t* edge_is_bnd) {
    if (!a || !a->computed) return 0u;
    const int rc = sb_guard([&] {
        if (row)
            SB_CUDA(cudaMemcpyAsync(row, a->row.ptr, sizeof(uint32_t) * ((size_t)a->n_nodes + 1), cudaMemcpyDeviceToHost,
                                    a->stream));
        if (neig)
            SB_CUDA(cudaMemcpyAsync(neig, a->neig.ptr, sizeof(uint32_t) * a->n_edges, cudaMemcpyDeviceToHost, a->stream));
        if (edge_is_bnd)
            SB_CUDA(cudaMemcpyAsync(edge_is_bnd, a->edge_is_bnd.ptr, a->n_edges, cudaMemcpyDeviceToHost, a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
    return rc ? 0u : a->n_edges;
}

SB_EXPORT uint32_t AlphaShape3D_get_boundary_nodes(const AlphaShape3D* a, uint8_t* is_bnd) {
    if (!a || !is_bnd || !a->computed) return 0u;
    const int rc = sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(is_bnd, a->node_is_bnd.ptr, a->n_nodes, cudaMemcpyDeviceToHost, a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
    return rc ? 0u : a->n_nodes;
}

// Per-star diagnostics in Morton order: nineig (star size incl. infinity
// ids), nkeep (kept local tets), candidate lists (n x 124, traversal order,
// entries past nineig-4 undefined).  Any pointer may be null.
SB_EXPORT int AlphaShape3D_get_stars(const AlphaShape3D* a, uint32_t* nineig, uint8_t* nkeep, uint32_t* cand) {
    if (!a || !a->computed) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const uint32_t n = a->n_nodes;
        if (nineig)
            SB_CUDA(cudaMemcpyAsync(nineig, a->nineig.ptr, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, a->stream));
        if (nkeep) SB_CUDA(cudaMemcpyAsync(nkeep, a->nkeep.ptr, n, cudaMemcpyDeviceToHost, a->stream));
        if (cand) {
            std::vector<uint32_t> ell((size_t)((n + 31) / 32) * sb::kCandMax * 32);
            SB_CUDA(cudaMemcpyAsync(ell.data(), a->cand.ptr, sizeof(uint32_t) * ell.size(), cudaMemcpyDeviceToHost,
                                    a->stream));
            SB_CUDA(cudaStreamSynchronize(a->stream));
            for (uint32_t i = 0; i < n; ++i)
                for (int j = 0; j < sb::kCandMax; ++j)
                    cand[(size_t)i * sb::kCandMax + j] = ell[sb::cand_at(i, (uint32_t)j)];
        }
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
}

// Device pointers of the resident outputs (for callers chaining kernels on
// the same GPU).  Valid until the next set_nodes/init/compute.
SB_EXPORT int AlphaShape3D_get_device_outputs(const AlphaShape3D* a, const void** obj_m, const void** elems,
                                              const void** row, const void** neig, const void** node_is_bnd) {
    if (!a || !a->computed) return (int)sb::ST_BAD_INPUT;
    if (obj_m) *obj_m = a->lbvh.obj_m.ptr;
    if (elems) *elems = a->elems.ptr;
    if (row) *row = a->row.ptr;
    if (neig) *neig = a->neig.ptr;
    if (node_is_bnd) *node_is_bnd = a->node_is_bnd.ptr;
    return 0;
}

SB_EXPORT int AlphaShape3D_set_profiling(AlphaShape3D* a, int on) {
    if (!a) return (int)sb::ST_BAD_INPUT;
    a->profiling = on != 0;
    return 0;
}

// Device milliseconds of the stages of the last init()+compute() with
// profiling on: {bbox+Morton+histogram, radix sort, gather+Karras+fit+infinity
// points, candidate search, star (fast stages), star (exact stage), scans and
// size read-back, compress}.
SB_EXPORT int AlphaShape3D_get_profile(AlphaShape3D* a, float* ms8) {
    if (!a || !ms8 || !a->profiling || !a->computed) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        a->collect_profile();
        static_assert(sb::AlphaShape3D::S_COUNT == 8, "ms8 holds one value per stage");
        for (int i = 0; i < sb::AlphaShape3D::S_COUNT; ++i) ms8[i] = a->stage_ms[i];
    });
}

// The same stages (at most count values); *written = how many.
SB_EXPORT int AlphaShape3D_get_profile_stages(AlphaShape3D* a, float* ms, uint32_t count, uint32_t* written) {
    if (!a || !ms || !a->profiling || !a->computed) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        a->collect_profile();
        const uint32_t k = std::min<uint32_t>(count, (uint32_t)sb::AlphaShape3D::S_COUNT);
        for (uint32_t i = 0; i < k; ++i) ms[i] = a->stage_ms[i];
        if (written) *written = k;
    });
}

SB_EXPORT int AlphaShape3D_set_work_counters(AlphaShape3D* a, int on) {
    if (!a) return (int)sb::ST_BAD_INPUT;
    a->count_work = on != 0;
    return 0;
}

// out2 = {stage-1 insphere tests, stage-2 FP64 evaluations} of the fast star
// pass of the last compute() run with work counters on.
SB_EXPORT int AlphaShape3D_get_work(AlphaShape3D* a, uint64_t* out2) {
    if (!a || !out2 || !a->computed || !a->count_work) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(out2, a->work.ptr, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, a->stream));
        SB_CUDA(cudaStreamSynchronize(a->stream));
    });
}

SB_EXPORT int AlphaShape3D_set_stream(AlphaShape3D* a, void* stream) {
    if (!a) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] { a->set_stream(static_cast<cudaStream_t>(stream)); });
}

SB_EXPORT int AlphaShape3D_synchronize(AlphaShape3D* a) {
    if (!a) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] { SB_CUDA(cudaStreamSynchronize(a->stream)); });
}

// Conflict decisions of the star kernel on host arrays (pts m x 5 x 3, ids
// m x 5); out receives the reference's 'det' per quintuple.  Test entry.
SB_EXPORT int stream_b200_conflict_batch(uint32_t m, const float* pts, const uint32_t* ids, float* out) {
    if (m == 0) return 0;
    if (!pts || !ids || !out) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        sb::DeviceBuffer<float> dp, dout;
        sb::DeviceBuffer<uint32_t> di, dst;
        dp.ensure(15 * (size_t)m);
        di.ensure(5 * (size_t)m);
        dout.ensure(m);
        dst.ensure(1);
        SB_CUDA(cudaMemcpy(dp.ptr, pts, sizeof(float) * 15 * (size_t)m, cudaMemcpyHostToDevice));
        SB_CUDA(cudaMemcpy(di.ptr, ids, sizeof(uint32_t) * 5 * (size_t)m, cudaMemcpyHostToDevice));
        SB_CUDA(cudaMemset(dst.ptr, 0, sizeof(uint32_t)));
        sb::conflict_batch_device(m, dp.ptr, di.ptr, dout.ptr, dst.ptr, 0);
        SB_CUDA(cudaMemcpy(out, dout.ptr, sizeof(float) * m, cudaMemcpyDeviceToHost));
    });
}

// ---------------------------------------------------------------- LBVH ----
// The reference exposes Sphere3DLBVH as a C++ type only (include/geometry/
// lbvh.hpp:50,62-362); these entry points give it a C boundary.
SB_EXPORT Sphere3DLBVH* Sphere3DLBVH_create(void) {
    Sphere3DLBVH* h = nullptr;
    sb_guard([&] { h = new Sphere3DLBVH; });
    return h;
}

SB_EXPORT void Sphere3DLBVH_destroy(Sphere3DLBVH* h) { sb_guard([&] { delete h; }); }

// xyzr: n x 4 host floats (centre, radius).  bits: 63 or 30.  fit_point: 1 =
// node boxes of the centres (the mesher's functor), 0 = of the spheres.
SB_EXPORT int Sphere3DLBVH_set_objects(Sphere3DLBVH* h, uint32_t n, const float* xyzr, int bits, int fit_point) {
    if (!h || !xyzr || n < 2 || (bits != 63 && bits != 30)) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        h->objs.ensure(n);
        SB_CUDA(cudaMemcpyAsync(h->objs.ptr, xyzr, sizeof(float4) * n, cudaMemcpyHostToDevice, h->stream));
        h->bvh.n = n;
        h->bvh.bits = bits;
        h->bvh.fit_point = fit_point != 0;
        SB_CUDA(cudaStreamSynchronize(h->stream));
    });
}

SB_EXPORT int Sphere3DLBVH_set_objects_device(Sphere3DLBVH* h, uint32_t n, const float* d_xyzr, int bits, int fit_point) {
    if (!h || !d_xyzr || n < 2 || (bits != 63 && bits != 30)) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        h->objs.ensure(n);
        SB_CUDA(cudaMemcpyAsync(h->objs.ptr, d_xyzr, sizeof(float4) * n, cudaMemcpyDeviceToDevice, h->stream));
        h->bvh.n = n;
        h->bvh.bits = bits;
        h->bvh.fit_point = fit_point != 0;
    });
}

// Enqueue the build on the handle's stream (asynchronous).
SB_EXPORT int Sphere3DLBVH_build(Sphere3DLBVH* h) {
    if (!h || h->bvh.n < 2) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemsetAsync(h->status.ptr, 0, sizeof(uint32_t), h->stream));
        h->marks.begin(h->stream);
        h->bvh.build(h->objs.ptr, h->bvh.n, h->stream, h->status.ptr, h->marks.on ? h : nullptr);
        h->marks.record();
    });
}

// Additive: record CUDA events between the build's stages (on = 1).
SB_EXPORT int Sphere3DLBVH_set_profiling(Sphere3DLBVH* h, int on) {
    if (!h) return (int)sb::ST_BAD_INPUT;
    h->marks.on = on != 0;
    return 0;
}
// Additive: stage times (ms) of the last profiled build: box + Morton codes,
// radix sort, gather, hierarchy + fit.  Returns the number written (<= cap).
SB_EXPORT uint32_t Sphere3DLBVH_get_profile(Sphere3DLBVH* h, float* ms, uint32_t cap) {
    if (!h || !ms) return 0u;
    uint32_t k = 0;
    sb_guard([&] { k = h->marks.elapsed(ms, cap); });
    return k;
}

SB_EXPORT int Sphere3DLBVH_synchronize(Sphere3DLBVH* h, uint32_t* status) {
    if (!h) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        uint32_t st = 0;
        SB_CUDA(cudaMemcpyAsync(&st, h->status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
        SB_CUDA(cudaStreamSynchronize(h->stream));
        if (status) *status = st;
    });
}

// Copy the build out (any pointer may be null): bb_glob[6], codes[n] (sorted),
// perm[n], sep[n-1], cil[n-1], leaf_parent[n], internal_parent[n-1],
// bboxes[(n-1) x 6], obj_m[n x 4].
SB_EXPORT int Sphere3DLBVH_get(Sphere3DLBVH* h, float* bb_glob, uint64_t* codes, uint32_t* perm, int32_t* sep,
                               uint8_t* cil, uint32_t* leaf_parent, uint32_t* internal_parent, float* bboxes,
                               float* obj_m) {
    if (!h || h->bvh.n < 2) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const uint32_t n = h->bvh.n;
        cudaStream_t s = h->stream;
        auto cp = [&](void* dst, const void* src, size_t bytes) {
            if (dst) SB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        };
        cp(bb_glob, h->bvh.bb_glob.ptr, 6 * sizeof(float));
        cp(codes, h->bvh.codes.ptr, 8 * (size_t)n);
        cp(perm, h->bvh.perm.ptr, 4 * (size_t)n);
        cp(sep, h->bvh.sep.ptr, 4 * (size_t)(n - 1));
        cp(cil, h->bvh.cil.ptr, (size_t)(n - 1));
        cp(leaf_parent, h->bvh.leaf_parent.ptr, 4 * (size_t)n);
        cp(internal_parent, h->bvh.internal_parent.ptr, 4 * (size_t)(n - 1));
        cp(obj_m, h->bvh.obj_m.ptr, 16 * (size_t)n);
        if (bboxes) {
            std::vector<sb::NodeBox> b(n - 1);
            SB_CUDA(cudaMemcpyAsync(b.data(), h->bvh.boxes.ptr, sizeof(sb::NodeBox) * (n - 1), cudaMemcpyDeviceToHost, s));
            SB_CUDA(cudaStreamSynchronize(s));
            for (uint32_t i = 0; i + 1 < n; ++i) {
                float* o = bboxes + 6 * (size_t)i;
                o[0] = b[i].lo.x; o[1] = b[i].lo.y; o[2] = b[i].lo.z;
                o[3] = b[i].hi.x; o[4] = b[i].hi.y; o[5] = b[i].hi.z;
            }
        }
        SB_CUDA(cudaStreamSynchronize(s));
    });
}

// --------------------------------------------------------------- TRBVH ----
// The reference exposes Sphere3DTRBVH (include/geometry/trbvh.hpp:55) as a C++
// type only; these entry points are additive.
SB_EXPORT Sphere3DTRBVH* Sphere3DTRBVH_create(void) {
    Sphere3DTRBVH* h = nullptr;
    sb_guard([&] { h = new Sphere3DTRBVH; });
    return h;
}

SB_EXPORT void Sphere3DTRBVH_destroy(Sphere3DTRBVH* h) { sb_guard([&] { delete h; }); }

// xyzr: n x 4 host floats.  treelet_size in [3, 8] (reference: 5); area3d 1 =
// half surface xy+yz+zx, 0 = the reference's ext_x*ext_y; rounds of
// restructuring (reference: 3, min sizes K, 2K, 4K; 0 = Apetrei build only).
SB_EXPORT int Sphere3DTRBVH_set_objects(Sphere3DTRBVH* h, uint32_t n, const float* xyzr, int treelet_size, int area3d,
                                        int rounds) {
    if (!h || !xyzr || n < 2 || treelet_size < 3 || treelet_size > sb::kTreeletMax || rounds < 0 || rounds > 8)
        return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        h->objs.ensure(n);
        SB_CUDA(cudaMemcpyAsync(h->objs.ptr, xyzr, sizeof(float4) * n, cudaMemcpyHostToDevice, h->stream));
        h->t.n = n;
        h->t.treelet_size = treelet_size;
        h->t.area3d = area3d != 0;
        h->t.rounds = rounds;
        SB_CUDA(cudaStreamSynchronize(h->stream));
    });
}

SB_EXPORT int Sphere3DTRBVH_build(Sphere3DTRBVH* h) {
    if (!h || h->t.n < 2) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemsetAsync(h->status.ptr, 0, sizeof(uint32_t), h->stream));
        h->marks.begin(h->stream);
        h->t.build(h->objs.ptr, h->t.n, h->stream, h->status.ptr, h->marks.on ? h : nullptr);
        h->marks.record();
    });
}

// Additive: record CUDA events between the build's stages (on = 1).
SB_EXPORT int Sphere3DTRBVH_set_profiling(Sphere3DTRBVH* h, int on) {
    if (!h) return (int)sb::ST_BAD_INPUT;
    h->marks.on = on != 0;
    return 0;
}
// Additive: stage times (ms) of the last profiled build: box + Morton codes,
// radix sort, gather, Apetrei build, treelet rounds.  Returns the number
// written (<= cap).
SB_EXPORT uint32_t Sphere3DTRBVH_get_profile(Sphere3DTRBVH* h, float* ms, uint32_t cap) {
    if (!h || !ms) return 0u;
    uint32_t k = 0;
    sb_guard([&] { k = h->marks.elapsed(ms, cap); });
    return k;
}

SB_EXPORT int Sphere3DTRBVH_synchronize(Sphere3DTRBVH* h, uint32_t* status) {
    if (!h) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        uint32_t st = 0;
        SB_CUDA(cudaMemcpyAsync(&st, h->status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
        SB_CUDA(cudaStreamSynchronize(h->stream));
        if (status) *status = st;
    });
}

// Copy out (any pointer may be NULL): child_left/right[n-1], range_min/max[n-1],
// parent[2n-1], bboxes[(2n-1) x 6], subtree_size[2n-1], sah[2n-1], root[1], obj_m[n x 4].
SB_EXPORT int Sphere3DTRBVH_get(Sphere3DTRBVH* h, uint32_t* child_left, uint32_t* child_right, uint32_t* range_min,
                                uint32_t* range_max, uint32_t* parent, float* bboxes, uint32_t* subtree_size, float* sah,
                                uint32_t* root, float* obj_m) {
    if (!h || h->t.n < 2) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const uint32_t n = h->t.n;
        const size_t m = 2 * (size_t)n - 1;
        cudaStream_t s = h->stream;
        auto cp = [&](void* dst, const void* src, size_t bytes) {
            if (dst) SB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        };
        cp(child_left, h->t.child_left.ptr, 4 * (size_t)(n - 1));
        cp(child_right, h->t.child_right.ptr, 4 * (size_t)(n - 1));
        cp(range_min, h->t.range_min.ptr, 4 * (size_t)(n - 1));
        cp(range_max, h->t.range_max.ptr, 4 * (size_t)(n - 1));
        cp(parent, h->t.parent.ptr, 4 * m);
        cp(subtree_size, h->t.subtree_size.ptr, 4 * m);
        cp(sah, h->t.sah.ptr, 4 * m);
        cp(root, h->t.root.ptr, 4);
        cp(obj_m, h->t.sorter.obj_m.ptr, 16 * (size_t)n);
        if (bboxes) {
            std::vector<sb::NodeBox> b(m);
            SB_CUDA(cudaMemcpyAsync(b.data(), h->t.boxes.ptr, sizeof(sb::NodeBox) * m, cudaMemcpyDeviceToHost, s));
            SB_CUDA(cudaStreamSynchronize(s));
            for (size_t i = 0; i < m; ++i) {
                float* o = bboxes + 6 * i;
                o[0] = b[i].lo.x; o[1] = b[i].lo.y; o[2] = b[i].lo.z;
                o[3] = b[i].hi.x; o[4] = b[i].hi.y; o[5] = b[i].hi.z;
            }
        }
        SB_CUDA(cudaStreamSynchronize(s));
    });
}

// Per object (Morton order), the number of other spheres overlapping it,
// found through the tree; out[n].
SB_EXPORT int Sphere3DTRBVH_count_overlaps(Sphere3DTRBVH* h, uint32_t* out) {
    if (!h || !out || h->t.n < 2) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        h->counts.ensure(h->t.n);
        h->t.count_overlaps(h->counts.ptr, h->stream);
        SB_CUDA(cudaMemcpyAsync(out, h->counts.ptr, 4 * (size_t)h->t.n, cudaMemcpyDeviceToHost, h->stream));
        SB_CUDA(cudaStreamSynchronize(h->stream));
    });
}

}  // extern "C"
