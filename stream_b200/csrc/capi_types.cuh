// The C handle types of the extern "C" boundary (opaque in stream_b200.h),
// shared by the capi_*.cu files.
#pragma once

#include <memory>
#include <stdexcept>
#include <vector>

#include "ashape3d.cuh"
#include "capi_common.cuh"
#include "fsai.cuh"
#include "numerics.cuh"
#include "stream_b200.h"

struct AlphaShape3D : sb::AlphaShape3D {};

struct HostCSR {
    uint32_t n = 0;
    std::vector<uint32_t> row, col;
    std::vector<float> val;
};

struct DeviceCSR {
    std::shared_ptr<sb::CsrF32> A = std::make_shared<sb::CsrF32>();
};

struct LinearSystem {
    uint32_t n = 0;
    std::shared_ptr<sb::CsrF32> A;  // shared with the DeviceCSR it was set from (linear_system.cpp:40)
    sb::DeviceBuffer<float> b;
};

struct PrecJacobi {
    std::shared_ptr<sb::CsrF32> A;
    uint32_t bad_rows = 0;  // rows without a usable diagonal (counted at creation)
};

struct ConjugateGradient {
    sb::CgWork w;
    sb::DeviceBuffer<float> x;
    uint32_t last_done = 0;  // termination of the last solve (0: none yet)
    cudaStream_t s = nullptr;
    ConjugateGradient() { SB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~ConjugateGradient() { if (s) cudaStreamDestroy(s); }
};

struct FsaiModel : sb::FsaiModel {};

// RHS modes {kx, ky, kz, a.k, phi} x nmodes (nmodes <= 8) of u = sum a sin(k.x + phi).
inline sb::DivModes sb_div_modes(const float* modes, int nmodes) {
    sb::DivModes dm;
    dm.count = modes ? nmodes : 0;
    for (int m = 0; m < dm.count; ++m) {
        dm.k[m][0] = modes[5 * m];
        dm.k[m][1] = modes[5 * m + 1];
        dm.k[m][2] = modes[5 * m + 2];
        dm.adotk[m] = modes[5 * m + 3];
        dm.phi[m] = modes[5 * m + 4];
    }
    return dm;
}

struct PoissonSystem {
    sb::CsrF64 A;
    sb::DeviceBuffer<double> b, x;
    sb::Assembly asmb;
    sb::CgWork w;
    sb::DeviceBuffer<float4> xyz;  // node coordinates (features of the learned preconditioner)
    bool has_xyz = false;
    sb::FsaiSystem fsai;
    FsaiModel* model = nullptr;
    double last_setup_ms = 0, last_infer_ms = 0, last_solve_ms = 0;
    uint32_t last_fallback = 0;
    cudaStream_t s = nullptr;

    PoissonSystem() { SB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~PoissonSystem() { if (s) cudaStreamDestroy(s); }
    PoissonSystem(const PoissonSystem&) = delete;
    PoissonSystem& operator=(const PoissonSystem&) = delete;

    const float4* coords() const { return has_xyz ? xyz.ptr : nullptr; }

    // P1 Laplacian on a computed mesh (its Morton order), coordinates kept for
    // the preconditioner's features, x = 0.  Dirichlet rows: the mesh's
    // free-surface nodes, or `dirichlet` (n flags) when given.  The mesh's work
    // must be complete or ordered before s.
    void assemble(const sb::AlphaShape3D& mesh, int rhs_kind, const sb::DivModes& dm,
                  const uint8_t* dirichlet = nullptr) {
        sb::assemble_p1_laplacian(mesh.n_nodes, mesh.lbvh.obj_m.ptr, mesh.elems.ptr, mesh.n_elems,
                                  dirichlet ? dirichlet : mesh.node_is_bnd.ptr, rhs_kind, dm, A, b, asmb, s);
        xyz.ensure(mesh.n_nodes);
        SB_CUDA(cudaMemcpyAsync(xyz.ptr, mesh.lbvh.obj_m.ptr, sizeof(float4) * mesh.n_nodes,
                                cudaMemcpyDeviceToDevice, s));
        has_xyz = true;
        fsai.invalidate();
        x.ensure(mesh.n_nodes);
        SB_CUDA(cudaMemsetAsync(x.ptr, 0, 8 * (size_t)mesh.n_nodes, s));
        SB_CUDA(cudaStreamSynchronize(s));
        if (asmb.overflow) throw std::runtime_error("assembly: row longer than 128 columns or node in > 256 elements");
    }

    // G of the attached model on this system, recomputed when the matrix or
    // the parameters changed.  Returns the set-up + inference ms that ran.
    double ensure_g() {
        double ms = 0.0;
        if (!fsai.prepared) {
            sb::fsai_prepare(A, coords(), fsai, s);
            last_setup_ms = fsai.setup_ms;
            ms += fsai.setup_ms;
        }
        if (fsai.g_ky || fsai.g_model != model || fsai.g_version != model->version) {
            sb::fsai_infer(*model, A, coords(), fsai, s);
            last_infer_ms = fsai.infer_ms;
            ms += fsai.infer_ms;
        }
        return ms;
    }

    // The Kolotilina-Yeremin G on this system, recomputed when the matrix
    // changed or g holds the model's G.  Returns the set-up + solve ms that ran.
    double ensure_ky() {
        double ms = 0.0;
        if (!fsai.prepared) {
            sb::fsai_prepare(A, coords(), fsai, s);
            last_setup_ms = fsai.setup_ms;
            ms += fsai.setup_ms;
        }
        if (!fsai.g_ky) {
            sb::fsai_ky(A, coords(), fsai, s);
            last_infer_ms = fsai.infer_ms;
            ms += fsai.infer_ms;
        }
        return ms;
    }

    // Solve from the current x (device).  method 0 FP64 Jacobi-PCG, 1 mixed
    // Jacobi refinement, 2 mixed learned-FSAI refinement (needs model), 3
    // mixed refinement with the Kolotilina-Yeremin FSAI.  The returned ms
    // includes the preconditioner's set-up and inference (or local solves).
    sb::SolveReport solve(int method, double rtol, uint32_t maxit, double inner_rtol) {
        sb::SolveReport r;
        double pre_ms = 0.0;
        if (method == 0) {
            r = sb::pcg_f64(A, b.ptr, x.ptr, rtol, maxit, w, s);
        } else if (method == 1) {
            r = sb::ir_mixed(A, b.ptr, x.ptr, rtol, maxit, inner_rtol, w, s);
        } else {
            if (method == 2 && !model) throw std::invalid_argument("solve: method 2 needs a model");
            pre_ms = method == 2 ? ensure_g() : ensure_ky();
            sb::FsaiOperator G{fsai.loff.ptr, fsai.lcol.ptr, fsai.lval.ptr, fsai.uoff.ptr, fsai.ucol.ptr, fsai.uval.ptr};
            r = sb::ir_fsai(A, b.ptr, x.ptr, rtol, maxit, inner_rtol, G, w, s);
        }
        last_solve_ms = r.ms;
        last_fallback = r.fallback;
        r.ms += pre_ms;
        return r;
    }
};
