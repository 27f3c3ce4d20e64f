// extern "C" boundary of the PFEM step loop: particles advected by an
// analytic Taylor-Green field, or moved by the fractional-step flow solver
// (gravity, viscosity, walls; PfemLoop_set_physics), remeshed (LBVH +
// alpha-shape Delaunay, free surface), P1 pressure system assembled and
// solved every step on one stream, with per-phase device timings.  The
// reference has no step loop.
#include <cmath>
#include <string>
#include <vector>

#include "capi_types.cuh"
#include "pfem.cuh"

struct PfemLoop {
    uint32_t n = 0;
    float alpha = 0.f;
    sb::DeviceBuffer<double> xyz;  // particle positions in particle order (FP64)
    sb::DeviceBuffer<float4> pts4; // (x, y, z, alpha) handed to the mesher
    sb::DeviceBuffer<double> p;    // last pressure in particle order: the next solve's initial guess
    bool has_p = false;
    sb::TaylorGreen flow{};
    sb::DivModes modes{};
    AlphaShape3D mesh;
    PoissonSystem ps;
    FsaiModel* model = nullptr;
    uint64_t steps_done = 0, fallbacks = 0;
    // fractional-step dynamics (off: Taylor-Green advection)
    bool physics = false;
    sb::FsParams fs{};
    sb::DeviceBuffer<double> u;                // particle velocities, particle order
    sb::DeviceBuffer<double> um, ustar, mass;  // mesh (Morton) order
    sb::DeviceBuffer<uint8_t> wall, dirichlet;
    PfemLoop() {
        flow.R[0] = flow.R[4] = flow.R[8] = 1.0;
        flow.k = 2.0 * M_PI;
        flow.amp = 0.5;
        mesh.set_stream(ps.s);
    }
};

namespace {

sb::TaylorGreen tg_from(const double* p) {
    sb::TaylorGreen f{};
    for (int i = 0; i < 9; ++i) f.R[i] = p[i];
    for (int i = 0; i < 3; ++i) f.c[i] = p[9 + i];
    f.k = p[12];
    f.amp = p[13];
    return f;
}

struct PhaseEvents {
    cudaEvent_t e[8] = {};
    PhaseEvents() {
        for (auto& x : e) SB_CUDA(cudaEventCreate(&x));
    }
    ~PhaseEvents() {
        for (auto& x : e)
            if (x) cudaEventDestroy(x);
    }
    float ms(int a, int b) const {
        float t = 0.f;
        SB_CUDA(cudaEventElapsedTime(&t, e[a], e[b]));
        return t;
    }
};

}  // namespace

extern "C" {

// Euler steps of a Taylor-Green field on host positions (n x 3 FP64, in
// place), computed on the GPU.  tg = {R[9] row-major, c[3], k, amp}.
SB_EXPORT int stream_b200_advect_taylor_green(uint32_t n, double* xyz, const double* tg, double dt, uint32_t steps) {
    if (!xyz || !tg || n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        sb::DeviceBuffer<double> d;
        d.ensure(3 * (size_t)n);
        SB_CUDA(cudaMemcpy(d.ptr, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
        sb::advect_taylor_green(n, d.ptr, tg_from(tg), dt, steps, 0.f, nullptr, 0);
        SB_CUDA(cudaMemcpy(xyz, d.ptr, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    });
}

SB_EXPORT PfemLoop* PfemLoop_create(void) {
    PfemLoop* p = nullptr;
    sb_guard([&] { p = new PfemLoop; });
    return p;
}

SB_EXPORT void PfemLoop_destroy(PfemLoop* L) { sb_guard([&] { delete L; }); }

SB_EXPORT int PfemLoop_set_particles(PfemLoop* L, uint32_t n, const double* xyz, float alpha) {
    if (!L || !xyz || n < 2 || !(alpha > 0)) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        L->n = n;
        L->alpha = alpha;
        L->xyz.ensure(3 * (size_t)n);
        L->pts4.ensure(n);
        L->p.ensure(n);
        L->u.ensure(3 * (size_t)n);
        L->has_p = false;
        SB_CUDA(cudaMemcpyAsync(L->xyz.ptr, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, L->ps.s));
        SB_CUDA(cudaMemsetAsync(L->u.ptr, 0, sizeof(double) * 3 * n, L->ps.s));
        SB_CUDA(cudaStreamSynchronize(L->ps.s));
    });
}

// Fractional-step dynamics instead of the Taylor-Green advection: params =
// {g[3], nu, rho, box lo[3], box hi[3]} (11 values; rho > 0, nu >= 0,
// lo < hi).  Velocities start at zero (PfemLoop_set_velocity).  NULL turns
// the dynamics off.
SB_EXPORT int PfemLoop_set_physics(PfemLoop* L, const double* params) {
    if (!L) return (int)sb::ST_BAD_INPUT;
    if (!params) {
        L->physics = false;
        return 0;
    }
    sb::FsParams f{};
    for (int k = 0; k < 3; ++k) {
        f.g[k] = params[k];
        f.lo[k] = params[5 + k];
        f.hi[k] = params[8 + k];
        if (!(f.lo[k] < f.hi[k]) || !std::isfinite(f.g[k])) return (int)sb::ST_BAD_INPUT;
    }
    f.nu = params[3];
    f.rho = params[4];
    if (!(f.rho > 0) || !(f.nu >= 0) || !std::isfinite(f.nu) || !std::isfinite(f.rho)) return (int)sb::ST_BAD_INPUT;
    L->fs = f;
    L->physics = true;
    return 0;
}

// Particle velocities (n x 3 FP64, particle order).
SB_EXPORT int PfemLoop_get_velocity(const PfemLoop* L, double* uvw) {
    if (!L || !uvw || L->n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(uvw, L->u.ptr, sizeof(double) * 3 * L->n, cudaMemcpyDeviceToHost, L->ps.s));
        SB_CUDA(cudaStreamSynchronize(L->ps.s));
    });
}

SB_EXPORT int PfemLoop_set_velocity(PfemLoop* L, const double* uvw) {
    if (!L || !uvw || L->n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(L->u.ptr, uvw, sizeof(double) * 3 * L->n, cudaMemcpyHostToDevice, L->ps.s));
        SB_CUDA(cudaStreamSynchronize(L->ps.s));
    });
}

SB_EXPORT int PfemLoop_get_particles(const PfemLoop* L, double* xyz) {
    if (!L || !xyz || L->n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(xyz, L->xyz.ptr, sizeof(double) * 3 * L->n, cudaMemcpyDeviceToHost, L->ps.s));
        SB_CUDA(cudaStreamSynchronize(L->ps.s));
    });
}

SB_EXPORT int PfemLoop_set_flow(PfemLoop* L, const double* tg) {
    if (!L || !tg) return (int)sb::ST_BAD_INPUT;
    L->flow = tg_from(tg);
    return 0;
}

SB_EXPORT int PfemLoop_set_rhs_modes(PfemLoop* L, const float* modes, int nmodes) {
    if (!L || nmodes < 0 || nmodes > 8 || (nmodes && !modes)) return (int)sb::ST_BAD_INPUT;
    L->modes = sb_div_modes(modes, nmodes);
    return 0;
}

SB_EXPORT int PfemLoop_set_fsai(PfemLoop* L, FsaiModel* m) {
    if (!L) return (int)sb::ST_BAD_INPUT;
    L->model = m;
    L->ps.model = m;
    return 0;
}

namespace {

void remesh(PfemLoop* L) {
    L->mesh.set_nodes_device(L->n, L->pts4.ptr);
    L->mesh.init();
    L->mesh.compute();
    L->mesh.read_counters();
    const uint32_t bad = L->mesh.last_status & (sb::ST_STACK_OVERFLOW | sb::ST_EXACT_OVERFLOW |
                                               sb::ST_LOOKBACK_TIMEOUT | sb::ST_CUDA_ERROR);
    if (bad) throw std::runtime_error("PfemLoop_step: remesh failed (status " + std::to_string(bad) + ")");
    if (L->mesh.n_nodes != L->n) throw std::runtime_error("PfemLoop_step: mesh nodes differ from particles");
}

// One fractional step (pfem.cuh): remesh the current positions, predictor,
// pressure solve on the new mesh, correction and particle move.
sb::SolveReport physics_step(PfemLoop* L, double dt, double rtol, PhaseEvents& ev) {
    cudaStream_t s = L->ps.s;
    const uint32_t n = L->n;
    L->fs.wall_tol = 0.5 * (double)L->alpha;  // wall nodes: within alpha / 2 of a box face
    SB_CUDA(cudaEventRecord(ev.e[0], s));
    sb::pack_particles(n, L->xyz.ptr, L->alpha, L->pts4.ptr, s);
    SB_CUDA(cudaEventRecord(ev.e[1], s));
    remesh(L);
    SB_CUDA(cudaEventRecord(ev.e[2], s));
    L->um.ensure(3 * (size_t)n);
    L->ustar.ensure(3 * (size_t)n);
    L->mass.ensure(n);
    L->wall.ensure(n);
    L->dirichlet.ensure(n);
    const float4* cm = L->mesh.lbvh.obj_m.ptr;
    const uint32_t* perm = L->mesh.lbvh.perm.ptr;
    sb::fs_gather(n, perm, L->u.ptr, cm, L->mesh.node_is_bnd.ptr, L->fs, L->um.ptr, L->wall.ptr, L->dirichlet.ptr, s);
    L->ps.assemble(L->mesh, 0, L->modes, L->dirichlet.ptr);
    SB_CUDA(cudaEventRecord(ev.e[3], s));
    const uint32_t* off = L->ps.asmb.off.ptr;
    const uint32_t* inc = L->ps.asmb.inc.ptr;
    sb::fs_predict(n, cm, L->mesh.elems.ptr, off, inc, L->um.ptr, L->wall.ptr, L->fs, dt, L->ustar.ptr, L->mass.ptr,
                   L->ps.b.ptr, L->dirichlet.ptr, s);
    SB_CUDA(cudaEventRecord(ev.e[4], s));
    if (L->has_p) sb::pressure_from_particles(n, perm, L->p.ptr, L->dirichlet.ptr, L->ps.x.ptr, s);
    const int method = L->model ? 2 : 0;
    if (method == 2) L->ps.ensure_g();
    SB_CUDA(cudaEventRecord(ev.e[5], s));
    const sb::SolveReport r = L->ps.solve(method, rtol, 100000u, 0.0);
    SB_CUDA(cudaEventRecord(ev.e[6], s));
    sb::fs_correct(n, cm, L->mesh.elems.ptr, off, inc, L->ps.x.ptr, L->mass.ptr, L->ustar.ptr, L->wall.ptr, perm,
                   L->fs, dt, L->alpha, L->u.ptr, L->xyz.ptr, L->pts4.ptr, s);
    sb::pressure_to_particles(n, perm, L->ps.x.ptr, L->p.ptr, s);
    L->has_p = true;
    SB_CUDA(cudaEventRecord(ev.e[7], s));
    SB_CUDA(cudaEventSynchronize(ev.e[7]));
    return r;
}

}  // namespace

SB_EXPORT int PfemLoop_step(PfemLoop* L, double dt, double rtol, double* report) {
    if (!L || L->n < 2 || !(rtol > 0) || !(dt > 0)) return (int)sb::ST_BAD_INPUT;
    if (L->physics)
        return sb_guard([&] {
            PhaseEvents ev;
            const sb::SolveReport r = physics_step(L, dt, rtol, ev);
            ++L->steps_done;
            L->fallbacks += r.fallback;
            if (report) {
                report[0] = ev.ms(0, 1) + ev.ms(3, 4) + ev.ms(6, 7);  // predictor, correction, particle move
                report[1] = ev.ms(1, 2);                             // remesh
                report[2] = ev.ms(2, 3);                             // assembly
                report[3] = ev.ms(4, 5);                             // preconditioner set-up + inference
                report[4] = ev.ms(5, 6);                             // solve
                report[5] = ev.ms(0, 7);                             // step
                report[6] = r.iterations;
                report[7] = r.fallback;
                report[8] = L->mesh.n_nodes;
                report[9] = L->mesh.n_elems;
                report[10] = r.relres;
                report[11] = r.converged;
            }
        });
    return sb_guard([&] {
        cudaStream_t s = L->ps.s;
        PhaseEvents ev;
        SB_CUDA(cudaEventRecord(ev.e[0], s));
        sb::advect_taylor_green(L->n, L->xyz.ptr, L->flow, dt, 1, L->alpha, L->pts4.ptr, s);
        SB_CUDA(cudaEventRecord(ev.e[1], s));
        remesh(L);
        SB_CUDA(cudaEventRecord(ev.e[2], s));
        L->ps.assemble(L->mesh, L->modes.count ? 1 : 0, L->modes);
        if (L->has_p)  // warm start: the previous step's pressure at the same particles
            sb::pressure_from_particles(L->n, L->mesh.lbvh.perm.ptr, L->p.ptr, L->mesh.node_is_bnd.ptr, L->ps.x.ptr, s);
        SB_CUDA(cudaEventRecord(ev.e[3], s));
        const int method = L->model ? 2 : 0;
        if (method == 2) L->ps.ensure_g();  // the assembly invalidated the previous step's preconditioner
        SB_CUDA(cudaEventRecord(ev.e[4], s));
        const sb::SolveReport r = L->ps.solve(method, rtol, 100000u, 0.0);
        sb::pressure_to_particles(L->n, L->mesh.lbvh.perm.ptr, L->ps.x.ptr, L->p.ptr, s);
        L->has_p = true;
        SB_CUDA(cudaEventRecord(ev.e[5], s));
        SB_CUDA(cudaEventSynchronize(ev.e[5]));
        ++L->steps_done;
        L->fallbacks += r.fallback;
        if (report) {
            report[0] = ev.ms(0, 1);   // advection
            report[1] = ev.ms(1, 2);   // remesh: LBVH + alpha shape + free surface
            report[2] = ev.ms(2, 3);   // assembly
            report[3] = ev.ms(3, 4);   // preconditioner set-up + inference
            report[4] = ev.ms(4, 5);   // solve
            report[5] = ev.ms(0, 5);   // step
            report[6] = r.iterations;
            report[7] = r.fallback;
            report[8] = L->mesh.n_nodes;
            report[9] = L->mesh.n_elems;
            report[10] = r.relres;
            report[11] = r.converged;
        }
    });
}

// Pressure of the last step in particle order (n values).
SB_EXPORT int PfemLoop_get_pressure(PfemLoop* L, double* p) {
    if (!L || !p || !L->has_p) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(p, L->p.ptr, sizeof(double) * L->n, cudaMemcpyDeviceToHost, L->ps.s));
        SB_CUDA(cudaStreamSynchronize(L->ps.s));
    });
}

// Initial guess of the next solve in particle order (n values), e.g. the
// pressure saved with a checkpoint.
SB_EXPORT int PfemLoop_set_pressure(PfemLoop* L, const double* p) {
    if (!L || !p || L->n == 0) return (int)sb::ST_BAD_INPUT;
    return sb_guard([&] {
        SB_CUDA(cudaMemcpyAsync(L->p.ptr, p, sizeof(double) * L->n, cudaMemcpyHostToDevice, L->ps.s));
        SB_CUDA(cudaStreamSynchronize(L->ps.s));
        L->has_p = true;
    });
}

// stats[2] = {steps done, steps that needed the Jacobi fallback}.
SB_EXPORT int PfemLoop_stats(const PfemLoop* L, uint64_t* stats) {
    if (!L || !stats) return (int)sb::ST_BAD_INPUT;
    stats[0] = L->steps_done;
    stats[1] = L->fallbacks;
    return 0;
}

// Borrowed handles of the current step's mesh and pressure system (valid
// until the next step or PfemLoop_destroy).
SB_EXPORT AlphaShape3D* PfemLoop_mesh(PfemLoop* L) { return L ? &L->mesh : nullptr; }
SB_EXPORT PoissonSystem* PfemLoop_system(PfemLoop* L) { return L ? &L->ps : nullptr; }

}  // extern "C"
