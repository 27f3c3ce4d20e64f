// extern "C" boundary for the numerics: the reference's CSR / linear system /
// Jacobi / CG handles (include/numerics/{csr,linear_system,preconditioner,
// solver}.hpp C blocks) and the additive FP64 / mixed-precision Poisson solve.
#include <cstring>
#include <memory>
#include <vector>

#include "capi_types.cuh"

namespace {
void upload_f32(sb::CsrF32& A, const HostCSR& h, cudaStream_t s) {
    A.n = h.n;
    A.nnz = (uint32_t)h.col.size();
    A.row.ensure(h.row.size());
    A.col.ensure(h.col.size());
    A.val.ensure(h.val.size());
    SB_CUDA(cudaMemcpyAsync(A.row.ptr, h.row.data(), 4 * h.row.size(), cudaMemcpyHostToDevice, s));
    if (!h.col.empty()) {
        SB_CUDA(cudaMemcpyAsync(A.col.ptr, h.col.data(), 4 * h.col.size(), cudaMemcpyHostToDevice, s));
        SB_CUDA(cudaMemcpyAsync(A.val.ptr, h.val.data(), 4 * h.val.size(), cudaMemcpyHostToDevice, s));
    }
    SB_CUDA(cudaStreamSynchronize(s));
}
}  // namespace

extern "C" {

// ---- reference numerics C ABI (src/numerics/*.cpp extern "C" blocks) --------
// csr.cpp:105-107
SB_EXPORT d_CSR* d_csr_create(void) {
    d_CSR* p = nullptr;
    sb_guard([&] { p = new DeviceCSR; });
    return p;
}
// csr.cpp:113-115
SB_EXPORT void d_csr_destroy(d_CSR* A) { sb_guard([&] { delete A; }); }
// csr.cpp:118-124 (nnz = row[n]; arrays are copied)
SB_EXPORT h_CSR* h_csr_create(uint32_t n, const uint32_t* row, const uint32_t* col, const float* val) {
    h_CSR* p = nullptr;
    sb_guard([&] {
        if (!row) throw std::invalid_argument("h_csr_create: null row");
        auto* h = new HostCSR;
        h->n = n;
        const uint32_t nnz = row[n];
        h->row.assign(row, row + n + 1);
        h->col.assign(col, col + nnz);
        h->val.assign(val, val + nnz);
        p = h;
    });
    return p;
}
// csr.cpp:126-128
SB_EXPORT void h_csr_destroy(h_CSR* A) { sb_guard([&] { delete A; }); }
// csr.cpp:109-111
SB_EXPORT void d_csr_h2d(d_CSR* dcsr, const h_CSR* hcsr) {
    if (!dcsr || !hcsr) return;
    sb_guard([&] {
        // A fresh device matrix, so linear systems already set keep theirs.
        dcsr->A = std::make_shared<sb::CsrF32>();
        upload_f32(*dcsr->A, *hcsr, 0);
    });
}
// linear_system.cpp:27-32
SB_EXPORT LinSys* LinSys_create(void) {
    LinSys* p = nullptr;
    sb_guard([&] { p = new LinearSystem; });
    return p;
}
// linear_system.cpp:34-36
SB_EXPORT void LinSys_destroy(LinSys* sys) { sb_guard([&] { delete sys; }); }
// linear_system.cpp:38-43: shares A's device arrays, copies b (host, A->n values).
SB_EXPORT void LinSys_set(LinSys* sys, const d_CSR* A, const float* b) {
    if (!sys || !A || !b) return;
    sb_guard([&] {
        sys->n = A->A->n;
        sys->A = A->A;
        sys->b.ensure(sys->n);
        SB_CUDA(cudaMemcpy(sys->b.ptr, b, 4 * (size_t)sys->n, cudaMemcpyHostToDevice));
    });
}
// preconditioner_jacobi.cpp:66-70.  Like the reference's init_device
// (:33-50), creation inspects the diagonal; rows without a usable one are
// counted (PrecJacobi_get_status) instead of leaving garbage.
SB_EXPORT PrecJacobi_st* PrecJacobi_create(const d_CSR* A) {
    PrecJacobi_st* p = nullptr;
    sb_guard([&] {
        auto* j = new PrecJacobi;
        j->A = A ? A->A : nullptr;
        if (j->A && j->A->n) {
            ConjugateGradient tmp;
            j->bad_rows = sb::count_bad_diagonal(*j->A, tmp.w, tmp.s);
        }
        p = j;
    });
    return p;
}
// Additive: 0 when every row has a nonzero diagonal entry with a finite
// inverse, else STREAM_ST_BAD_INPUT with the number of such rows in *bad_rows.
SB_EXPORT int PrecJacobi_get_status(const PrecJacobi_st* prec, uint32_t* bad_rows) {
    if (!prec) return (int)sb::ST_BAD_INPUT;
    if (bad_rows) *bad_rows = prec->bad_rows;
    return prec->bad_rows ? (int)sb::ST_BAD_INPUT : 0;
}
// preconditioner_jacobi.cpp:72-74
SB_EXPORT void PrecJacobi_destroy(PrecJacobi_st* prec) { sb_guard([&] { delete prec; }); }
// conjugate_gradient.cpp:215-217
SB_EXPORT SolverCG* SolverCG_create(void) {
    SolverCG* p = nullptr;
    sb_guard([&] { p = new ConjugateGradient; });
    return p;
}
// conjugate_gradient.cpp:219-221
SB_EXPORT void SolverCG_destroy(SolverCG* solver) { sb_guard([&] { delete solver; }); }

static uint32_t solve_ref(SolverCG* solver, const LinSys* sys, bool jacobi, float* x) {
    uint32_t it = 0;
    sb_guard([&] {
        if (!solver || !sys || !sys->A || !x) throw std::invalid_argument("SolverCG: null argument");
        const uint32_t n = sys->n;
        solver->x.ensure(n);
        SB_CUDA(cudaMemcpyAsync(solver->x.ptr, x, 4 * (size_t)n, cudaMemcpyHostToDevice, solver->s));
        solver->last_done = 0;
        it = sb::cg_f32_reference(*sys->A, sys->b.ptr, solver->x.ptr, jacobi, solver->w, solver->s,
                                  &solver->last_done);
        SB_CUDA(cudaMemcpyAsync(x, solver->x.ptr, 4 * (size_t)n, cudaMemcpyDeviceToHost, solver->s));
        SB_CUDA(cudaStreamSynchronize(solver->s));
    });
    return it;
}
// conjugate_gradient.cpp:223-229: Jacobi-PCG, x host in/out, returns the iteration counter.
SB_EXPORT uint32_t SolverCG_jacobi_solve(SolverCG* solver, const LinSys* sys, const PrecJacobi_st* prec, float* x) {
    (void)prec;  // the Jacobi diagonal is taken from the system matrix, as PrecJacobi_create does
    return solve_ref(solver, sys, true, x);
}
// conjugate_gradient.cpp:231-237: unpreconditioned CG.
SB_EXPORT uint32_t SolverCG_solve(SolverCG* solver, const LinSys* sys, float* x) { return solve_ref(solver, sys, false, x); }
// Additive: how the last solve ended: 1 the reference's stopping rule
// (sqrt(r.z) <= 1e-6), 2 its 10,000-iteration cap, 3 a non-finite r.z
// (breakdown, e.g. a zero diagonal), 0 no completed solve.
SB_EXPORT int SolverCG_get_termination(const SolverCG* solver) { return solver ? (int)solver->last_done : 0; }

// ---- additive: FP64 / mixed Poisson systems ----------------------------------
SB_EXPORT PoissonSystem* PoissonSystem_create(void) {
    PoissonSystem* p = nullptr;
    sb_guard([&] { p = new PoissonSystem; });
    return p;
}
SB_EXPORT void PoissonSystem_destroy(PoissonSystem* ps) { sb_guard([&] { delete ps; }); }

SB_EXPORT int PoissonSystem_assemble(PoissonSystem* ps, const AlphaShape3D* mesh, int rhs_kind, const float* modes,
                                     int nmodes) {
    if (!ps || !mesh || !mesh->computed || (rhs_kind != 0 && rhs_kind != 1) || nmodes < 0 || nmodes > 8 ||
        (rhs_kind == 1 && nmodes > 0 && !modes))
        return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaStreamSynchronize(mesh->stream));
        ps->assemble(*mesh, rhs_kind, sb_div_modes(rhs_kind == 1 ? modes : nullptr, rhs_kind == 1 ? nmodes : 0));
    });
}

SB_EXPORT int PoissonSystem_set_csr(PoissonSystem* ps, uint32_t n, const uint32_t* row, const uint32_t* col,
                                    const double* val, const double* b) {
    if (!ps || !row || !col || !val || !b || n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const uint32_t nnz = row[n];
        ps->A.n = n;
        ps->A.nnz = nnz;
        ps->A.row.ensure((size_t)n + 1);
        ps->A.col.ensure(nnz);
        ps->A.val.ensure(nnz);
        ps->A.invalidate_derived();
        ps->has_xyz = false;
        ps->fsai.invalidate();
        ps->b.ensure(n);
        ps->x.ensure(n);
        SB_CUDA(cudaMemcpyAsync(ps->A.row.ptr, row, 4 * ((size_t)n + 1), cudaMemcpyHostToDevice, ps->s));
        SB_CUDA(cudaMemcpyAsync(ps->A.col.ptr, col, 4 * (size_t)nnz, cudaMemcpyHostToDevice, ps->s));
        SB_CUDA(cudaMemcpyAsync(ps->A.val.ptr, val, 8 * (size_t)nnz, cudaMemcpyHostToDevice, ps->s));
        SB_CUDA(cudaMemcpyAsync(ps->b.ptr, b, 8 * (size_t)n, cudaMemcpyHostToDevice, ps->s));
        SB_CUDA(cudaMemsetAsync(ps->x.ptr, 0, 8 * (size_t)n, ps->s));
        SB_CUDA(cudaStreamSynchronize(ps->s));
    });
}

SB_EXPORT int PoissonSystem_get_size(const PoissonSystem* ps, uint32_t* n, uint32_t* nnz) {
    if (!ps) return (int)sb::ST_BAD_INPUT;
    if (n) *n = ps->A.n;
    if (nnz) *nnz = ps->A.nnz;
    return 0;
}

SB_EXPORT int PoissonSystem_get_csr(const PoissonSystem* ps, uint32_t* row, uint32_t* col, double* val, double* b) {
    if (!ps || ps->A.n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const uint32_t n = ps->A.n, nnz = ps->A.nnz;
        if (row) SB_CUDA(cudaMemcpyAsync(row, ps->A.row.ptr, 4 * ((size_t)n + 1), cudaMemcpyDeviceToHost, ps->s));
        if (col) SB_CUDA(cudaMemcpyAsync(col, ps->A.col.ptr, 4 * (size_t)nnz, cudaMemcpyDeviceToHost, ps->s));
        if (val) SB_CUDA(cudaMemcpyAsync(val, ps->A.val.ptr, 8 * (size_t)nnz, cudaMemcpyDeviceToHost, ps->s));
        if (b) SB_CUDA(cudaMemcpyAsync(b, ps->b.ptr, 8 * (size_t)n, cudaMemcpyDeviceToHost, ps->s));
        SB_CUDA(cudaStreamSynchronize(ps->s));
    });
}

// method 0: FP64 Jacobi-PCG; 1: mixed iterative refinement (FP32 inner
// Jacobi-PCG to inner_rtol, <= 0 for the automatic schedule, FP64 residual); 2: mixed iterative refinement
// with the learned FSAI preconditioner (PoissonSystem_set_fsai), Jacobi-PCG
// fallback on stagnation; 3: the same refinement with the Kolotilina-Yeremin
// FSAI on A's lower pattern (exact local solves, no model).  x: host FP64 initial guess and result (NULL: start
// from zero, result kept on the device).  report[6] = {iterations, outer
// steps, true relative residual, device ms (for method 2 including the
// preconditioner's set-up and inference when they ran), converged, fallback}.
SB_EXPORT int PoissonSystem_solve(PoissonSystem* ps, int method, double rtol, uint32_t maxit, double inner_rtol,
                                  double* x, double* report) {
    if (!ps || ps->A.n == 0 || method < 0 || method > 3 || !(rtol > 0)) return (int)sb::ST_BAD_INPUT;
    if (method == 2 && !ps->model) {
        sb::last_error_text() = "PoissonSystem_solve: method 2 needs a model (PoissonSystem_set_fsai)";
        return (int)sb::ST_BAD_INPUT;
    }
    return sb_guard([&] {
        const uint32_t n = ps->A.n;
        if (x) SB_CUDA(cudaMemcpyAsync(ps->x.ptr, x, 8 * (size_t)n, cudaMemcpyHostToDevice, ps->s));
        else SB_CUDA(cudaMemsetAsync(ps->x.ptr, 0, 8 * (size_t)n, ps->s));
        const sb::SolveReport r = ps->solve(method, rtol, maxit, inner_rtol);  // inner_rtol <= 0: automatic
        if (x) SB_CUDA(cudaMemcpyAsync(x, ps->x.ptr, 8 * (size_t)n, cudaMemcpyDeviceToHost, ps->s));
        SB_CUDA(cudaStreamSynchronize(ps->s));
        if (report) {
            report[0] = r.iterations;
            report[1] = r.outer;
            report[2] = r.relres;
            report[3] = r.ms;
            report[4] = r.converged;
            report[5] = r.fallback;
        }
    });
}

SB_EXPORT int PoissonSystem_get_solution(const PoissonSystem* ps, double* x) {
    if (!ps || !x || ps->A.n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(x, ps->x.ptr, 8 * (size_t)ps->A.n, cudaMemcpyDeviceToHost, ps->s));
        SB_CUDA(cudaStreamSynchronize(ps->s));
    });
}

SB_EXPORT int PoissonSystem_assembly_stats(const PoissonSystem* ps, uint32_t* isolated) {
    if (!ps) return (int)sb::ST_BAD_INPUT;
    if (isolated) *isolated = ps->asmb.n_isolated;
    return 0;
}

// ---- additive: learned FSAI preconditioner -------------------------------------
SB_EXPORT uint32_t FsaiModel_param_count(void) { return sb::kFsaiParamCount; }

SB_EXPORT FsaiModel* FsaiModel_create(void) {
    FsaiModel* p = nullptr;
    sb_guard([&] { p = new FsaiModel; });
    return p;
}
SB_EXPORT void FsaiModel_destroy(FsaiModel* m) { sb_guard([&] { delete m; }); }

SB_EXPORT int FsaiModel_set_params(FsaiModel* m, const float* params, uint32_t count) {
    if (!m || !params || count != sb::kFsaiParamCount) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemcpy(m->params.ptr, params, sizeof(float) * count, cudaMemcpyHostToDevice));
        ++m->version;
        m->packed = false;
    });
}

SB_EXPORT int FsaiModel_get_params(const FsaiModel* m, float* params, uint32_t count) {
    if (!m || !params || count != sb::kFsaiParamCount) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] { SB_CUDA(cudaMemcpy(params, m->params.ptr, sizeof(float) * count, cudaMemcpyDeviceToHost)); });
}

SB_EXPORT int FsaiModel_reset_optimizer(FsaiModel* m) {
    if (!m) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemset(m->m.ptr, 0, sizeof(float) * sb::kFsaiParamCount));
        SB_CUDA(cudaMemset(m->v.ptr, 0, sizeof(float) * sb::kFsaiParamCount));
        m->adam_t = 0;
    });
}

SB_EXPORT int FsaiModel_set_loss(FsaiModel* m, uint32_t kind) {
    if (!m || (kind != sb::kFsaiLossResidual && kind != sb::kFsaiLossKaporin)) return (int)sb::ST_BAD_INPUT;
    m->loss_kind = kind;
    return (int)sb::ST_OK;
}

SB_EXPORT int FsaiModel_set_base(FsaiModel* m, uint32_t base) {
    if (!m || (base != sb::kFsaiBaseNone && base != sb::kFsaiBaseKy)) return (int)sb::ST_BAD_INPUT;
    if (m->base != base) {
        m->base = base;
        ++m->version;  // attached systems rebuild G
    }
    return (int)sb::ST_OK;
}

SB_EXPORT int FsaiModel_get_base(const FsaiModel* m, uint32_t* base) {
    if (!m || !base) return (int)sb::ST_BAD_INPUT;
    *base = m->base;
    return (int)sb::ST_OK;
}

SB_EXPORT int FsaiModel_loss_grad(FsaiModel* m, PoissonSystem* ps, uint64_t seed, const float* probes, double* loss,
                                  float* grad) {
    if (!m || !ps || ps->A.n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const double L = sb::fsai_loss_grad(*m, ps->A, ps->coords(), ps->fsai, seed, probes, ps->s);
        if (loss) *loss = L;
        if (grad) {
            SB_CUDA(cudaMemcpyAsync(grad, m->grad.ptr, sizeof(float) * sb::kFsaiParamCount, cudaMemcpyDeviceToHost,
                                    ps->s));
            SB_CUDA(cudaStreamSynchronize(ps->s));
        }
    });
}

SB_EXPORT int FsaiModel_train_step(FsaiModel* m, PoissonSystem* ps, uint64_t seed, float lr, float clip,
                                   double* loss) {
    if (!m || !ps || ps->A.n == 0 || !(lr > 0)) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const double L = sb::fsai_loss_grad(*m, ps->A, ps->coords(), ps->fsai, seed, nullptr, ps->s);
        sb::fsai_adam(*m, lr, clip, ps->s);
        SB_CUDA(cudaStreamSynchronize(ps->s));
        if (loss) *loss = L;
    });
}

// One Adam step on the mean loss of count systems (probes seeded seed + i).
SB_EXPORT int FsaiModel_train_batch(FsaiModel* m, PoissonSystem* const* systems, uint32_t count, uint64_t seed,
                                    float lr, float clip, double* loss) {
    if (!m || !systems || count == 0 || !(lr > 0)) return (int)sb::ST_BAD_INPUT;
    for (uint32_t i = 0; i < count; ++i)
        if (!systems[i] || systems[i]->A.n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        double L = 0.0;
        cudaStream_t s = systems[0]->s;
        for (uint32_t i = 0; i < count; ++i) {
            PoissonSystem* ps = systems[i];
            L += sb::fsai_loss_grad(*m, ps->A, ps->coords(), ps->fsai, seed + i, nullptr, ps->s);
            sb::fsai_accumulate(*m, 1.0f / (float)count, i == 0, i + 1 == count, ps->s);
            SB_CUDA(cudaStreamSynchronize(ps->s));  // the next system reuses the model's gradient buffer
        }
        sb::fsai_adam(*m, lr, clip, s);
        SB_CUDA(cudaStreamSynchronize(s));
        if (loss) *loss = L / count;
    });
}

SB_EXPORT int PoissonSystem_set_coords(PoissonSystem* ps, const double* xyz) {
    if (!ps || !xyz || ps->A.n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        const uint32_t n = ps->A.n;
        std::vector<float4> h(n);
        for (uint32_t i = 0; i < n; ++i)
            h[i] = make_float4((float)xyz[3 * i], (float)xyz[3 * i + 1], (float)xyz[3 * i + 2], 0.f);
        ps->xyz.ensure(n);
        SB_CUDA(cudaMemcpyAsync(ps->xyz.ptr, h.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, ps->s));
        SB_CUDA(cudaStreamSynchronize(ps->s));
        ps->has_xyz = true;
        ps->fsai.invalidate();
    });
}

SB_EXPORT int PoissonSystem_set_fsai(PoissonSystem* ps, FsaiModel* m) {
    if (!ps) return (int)sb::ST_BAD_INPUT;
    ps->model = m;
    ps->fsai.invalidate();  // the next method-2 solve builds the preconditioner afresh
    return 0;
}

SB_EXPORT int PoissonSystem_get_fsai(PoissonSystem* ps, float* g, float* features, uint32_t* n_lower) {
    if (!ps || ps->A.n == 0 || (g && !ps->model)) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        if (!ps->fsai.prepared) sb::fsai_prepare(ps->A, ps->coords(), ps->fsai, ps->s);
        if (ps->fsai.error) throw std::runtime_error("fsai: the matrix needs a positive diagonal and sorted columns");
        if (n_lower) *n_lower = ps->fsai.n_edges;
        if (g) {
            ps->ensure_g();
            SB_CUDA(cudaMemcpyAsync(g, ps->fsai.g.ptr, sizeof(float) * ps->A.nnz, cudaMemcpyDeviceToHost, ps->s));
        }
        if (features) {
            sb::DeviceBuffer<float> f;
            f.ensure((size_t)ps->fsai.n_edges * sb::kFsaiNF);
            sb::fsai_features(ps->A, ps->coords(), ps->fsai, f.ptr, ps->s,
                              ps->model && ps->model->base == sb::kFsaiBaseKy);
            SB_CUDA(cudaMemcpyAsync(features, f.ptr, sizeof(float) * sb::kFsaiNF * ps->fsai.n_edges,
                                    cudaMemcpyDeviceToHost, ps->s));
            SB_CUDA(cudaStreamSynchronize(ps->s));
        }
        SB_CUDA(cudaStreamSynchronize(ps->s));
    });
}

// Additive: the Kolotilina-Yeremin G of method 3 (built if needed), aligned
// with the CSR like PoissonSystem_get_fsai, and the rows it left diagonal.
SB_EXPORT int PoissonSystem_get_ky(PoissonSystem* ps, float* g, uint32_t* diag_rows) {
    if (!ps || ps->A.n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        ps->ensure_ky();
        if (g) SB_CUDA(cudaMemcpyAsync(g, ps->fsai.g.ptr, sizeof(float) * ps->A.nnz, cudaMemcpyDeviceToHost, ps->s));
        if (diag_rows) *diag_rows = ps->fsai.ky_diag_rows;
        SB_CUDA(cudaStreamSynchronize(ps->s));
    });
}

// stats[4] = {set-up ms, inference ms, fallback of the last solve, lower edges}
SB_EXPORT int PoissonSystem_fsai_stats(const PoissonSystem* ps, double* stats) {
    if (!ps || !stats) return (int)sb::ST_BAD_INPUT;
    stats[0] = ps->last_setup_ms;
    stats[1] = ps->last_infer_ms;
    stats[2] = ps->last_fallback;
    stats[3] = ps->fsai.n_edges;
    return 0;
}

}  // extern "C"
