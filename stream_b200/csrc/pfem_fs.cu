// Fractional-step PFEM update on the P1 mesh of the particles (see pfem.cuh).
#include "pfem.cuh"

namespace sb {
namespace {

__device__ __forceinline__ double3 d3(const float4 v) { return make_double3(v.x, v.y, v.z); }
__device__ __forceinline__ double3 sub(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 cross(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Gradients of the four P1 basis functions and the volume of tet t (the
// same geometry as the assembly of the stiffness matrix); false when flat.
__device__ __forceinline__ bool tet_geometry(const float4* __restrict__ cm, const uint4 t, double3 g[4], double& vol) {
    const double3 x0 = d3(cm[t.x]), x1 = d3(cm[t.y]), x2 = d3(cm[t.z]), x3 = d3(cm[t.w]);
    const double3 e1 = sub(x1, x0), e2 = sub(x2, x0), e3 = sub(x3, x0);
    const double det = dot(e1, cross(e2, e3));
    if (det == 0.0) return false;
    const double inv = 1.0 / det;
    g[1] = cross(e2, e3);
    g[2] = cross(e3, e1);
    g[3] = cross(e1, e2);
    for (int k = 1; k < 4; ++k) g[k] = make_double3(g[k].x * inv, g[k].y * inv, g[k].z * inv);
    g[0] = make_double3(-(g[1].x + g[2].x + g[3].x), -(g[1].y + g[2].y + g[3].y), -(g[1].z + g[2].z + g[3].z));
    vol = fabs(det) / 6.0;
    return true;
}

__device__ __forceinline__ void zero_normals(uint32_t wall, double3& u) {
    if (wall & 0x03u) u.x = 0.0;
    if (wall & 0x0cu) u.y = 0.0;
    if (wall & 0x30u) u.z = 0.0;
}

// Node m of the mesh (Morton order): its particle's velocity, the walls it
// touches (bit 2k: below lo[k] + tol, bit 2k+1: above hi[k] - tol) and its
// pressure boundary condition (Dirichlet p = 0 on the free surface away from
// the walls; wall nodes keep the natural condition).
__global__ void k_fs_gather(uint32_t n, const uint32_t* __restrict__ perm, const double* __restrict__ u_p,
                            const float4* __restrict__ cm, const uint8_t* __restrict__ is_bnd, FsParams P,
                            double* __restrict__ um, uint8_t* __restrict__ wall, uint8_t* __restrict__ dirichlet) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const uint32_t q = perm[m];
    um[3 * (size_t)m] = u_p[3 * (size_t)q];
    um[3 * (size_t)m + 1] = u_p[3 * (size_t)q + 1];
    um[3 * (size_t)m + 2] = u_p[3 * (size_t)q + 2];
    const float4 c = cm[m];
    const double x[3] = {c.x, c.y, c.z};
    uint32_t w = 0;
    for (int k = 0; k < 3; ++k) {
        if (x[k] < P.lo[k] + P.wall_tol) w |= 1u << (2 * k);
        if (x[k] > P.hi[k] - P.wall_tol) w |= 2u << (2 * k);
    }
    wall[m] = (uint8_t)w;
    dirichlet[m] = (is_bnd[m] && !w) ? 1 : 0;
}

// Predictor: lumped mass M_i = sum vol/4 and the viscous term (K u)_i =
// sum vol grad(phi_i) . grad(u) over the incident elements;
// u* = u + dt (g - nu (K u)_i / M_i), normal components zeroed at walls.
__global__ void __launch_bounds__(128) k_fs_predict(uint32_t n, const float4* __restrict__ cm,
                                                    const uint4* __restrict__ el, const uint32_t* __restrict__ off,
                                                    const uint32_t* __restrict__ inc, const double* __restrict__ um,
                                                    const uint8_t* __restrict__ wall, FsParams P, double dt,
                                                    double* __restrict__ ustar, double* __restrict__ mass) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double M = 0.0, ku[3] = {0.0, 0.0, 0.0};
    for (uint32_t a = off[i]; a < off[i + 1]; ++a) {
        const uint4 t = el[inc[a]];
        double3 g[4];
        double vol;
        if (!tet_geometry(cm, t, g, vol)) continue;
        const uint32_t v[4] = {t.x, t.y, t.z, t.w};
        int li = 0;
        for (int k = 0; k < 4; ++k) if (v[k] == i) li = k;
        M += 0.25 * vol;
        for (int k = 0; k < 4; ++k) {
            const double kik = vol * dot(g[li], g[k]);
            for (int c = 0; c < 3; ++c) ku[c] += kik * um[3 * (size_t)v[k] + c];
        }
    }
    double3 u = make_double3(um[3 * (size_t)i], um[3 * (size_t)i + 1], um[3 * (size_t)i + 2]);
    const double s = M > 0.0 ? P.nu / M : 0.0;
    u.x += dt * (P.g[0] - s * ku[0]);
    u.y += dt * (P.g[1] - s * ku[1]);
    u.z += dt * (P.g[2] - s * ku[2]);
    zero_normals(wall[i], u);
    ustar[3 * (size_t)i] = u.x;
    ustar[3 * (size_t)i + 1] = u.y;
    ustar[3 * (size_t)i + 2] = u.z;
    mass[i] = M;
}

// Pressure load b_i = -(rho/dt) sum vol/4 div(u*) over the incident elements;
// 0 on Dirichlet rows and on nodes without elements (as the assembly's rows).
__global__ void __launch_bounds__(128) k_fs_rhs(uint32_t n, const float4* __restrict__ cm, const uint4* __restrict__ el,
                                                const uint32_t* __restrict__ off, const uint32_t* __restrict__ inc,
                                                const double* __restrict__ ustar, const uint8_t* __restrict__ dirichlet,
                                                double rho_over_dt, double* __restrict__ b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (dirichlet[i] || off[i + 1] == off[i]) {
        b[i] = 0.0;
        return;
    }
    double s = 0.0;
    for (uint32_t a = off[i]; a < off[i + 1]; ++a) {
        const uint4 t = el[inc[a]];
        double3 g[4];
        double vol;
        if (!tet_geometry(cm, t, g, vol)) continue;
        const uint32_t v[4] = {t.x, t.y, t.z, t.w};
        double div = 0.0;
        for (int k = 0; k < 4; ++k)
            div += dot(g[k], make_double3(ustar[3 * (size_t)v[k]], ustar[3 * (size_t)v[k] + 1], ustar[3 * (size_t)v[k] + 2]));
        s += 0.25 * vol * div;
    }
    b[i] = -rho_over_dt * s;
}

// Correction u = u* - (dt/rho) grad p (grad p lumped: sum vol/4 grad p_e / M_i),
// normal components zeroed at walls; then the particle moves by dt u and is
// kept inside the box (a particle that leaves it is put back on the wall and
// loses its normal velocity).  Writes the particle's velocity, position and
// the mesher's float4 in particle order.
__global__ void __launch_bounds__(128) k_fs_correct(uint32_t n, const float4* __restrict__ cm,
                                                    const uint4* __restrict__ el, const uint32_t* __restrict__ off,
                                                    const uint32_t* __restrict__ inc, const double* __restrict__ p,
                                                    const double* __restrict__ mass, const double* __restrict__ ustar,
                                                    const uint8_t* __restrict__ wall, const uint32_t* __restrict__ perm,
                                                    FsParams P, double dt, double dt_over_rho, float alpha,
                                                    double* __restrict__ u_p, double* __restrict__ xyz_p,
                                                    float4* __restrict__ pts4) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double gp[3] = {0.0, 0.0, 0.0};
    for (uint32_t a = off[i]; a < off[i + 1]; ++a) {
        const uint4 t = el[inc[a]];
        double3 g[4];
        double vol;
        if (!tet_geometry(cm, t, g, vol)) continue;
        const uint32_t v[4] = {t.x, t.y, t.z, t.w};
        double3 ge = make_double3(0.0, 0.0, 0.0);
        for (int k = 0; k < 4; ++k) {
            const double pk = p[v[k]];
            ge.x += pk * g[k].x;
            ge.y += pk * g[k].y;
            ge.z += pk * g[k].z;
        }
        gp[0] += 0.25 * vol * ge.x;
        gp[1] += 0.25 * vol * ge.y;
        gp[2] += 0.25 * vol * ge.z;
    }
    const double M = mass[i];
    const double s = M > 0.0 ? dt_over_rho / M : 0.0;
    double3 u = make_double3(ustar[3 * (size_t)i] - s * gp[0], ustar[3 * (size_t)i + 1] - s * gp[1],
                             ustar[3 * (size_t)i + 2] - s * gp[2]);
    zero_normals(wall[i], u);
    const uint32_t q = perm[i];
    double x[3] = {xyz_p[3 * (size_t)q] + dt * u.x, xyz_p[3 * (size_t)q + 1] + dt * u.y,
                   xyz_p[3 * (size_t)q + 2] + dt * u.z};
    double uu[3] = {u.x, u.y, u.z};
    for (int k = 0; k < 3; ++k) {
        if (x[k] < P.lo[k]) { x[k] = P.lo[k]; uu[k] = 0.0; }
        if (x[k] > P.hi[k]) { x[k] = P.hi[k]; uu[k] = 0.0; }
        u_p[3 * (size_t)q + k] = uu[k];
        xyz_p[3 * (size_t)q + k] = x[k];
    }
    pts4[q] = make_float4((float)x[0], (float)x[1], (float)x[2], alpha);
}

__global__ void k_pack_particles(uint32_t n, const double* __restrict__ xyz, float alpha, float4* __restrict__ out4) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out4[i] = make_float4((float)xyz[3 * (size_t)i], (float)xyz[3 * (size_t)i + 1], (float)xyz[3 * (size_t)i + 2], alpha);
}

}  // namespace

void pack_particles(uint32_t n, const double* xyz, float alpha, float4* out4, cudaStream_t s) {
    if (n == 0) return;
    k_pack_particles<<<grid_for(n, 256), 256, 0, s>>>(n, xyz, alpha, out4);
    SB_LAUNCH_CHECK();
}

void fs_gather(uint32_t n, const uint32_t* perm, const double* u_p, const float4* cm, const uint8_t* is_bnd,
               const FsParams& P, double* um, uint8_t* wall, uint8_t* dirichlet, cudaStream_t s) {
    if (n == 0) return;
    k_fs_gather<<<grid_for(n, 256), 256, 0, s>>>(n, perm, u_p, cm, is_bnd, P, um, wall, dirichlet);
    SB_LAUNCH_CHECK();
}

void fs_predict(uint32_t n, const float4* cm, const uint4* el, const uint32_t* off, const uint32_t* inc,
                const double* um, const uint8_t* wall, const FsParams& P, double dt, double* ustar, double* mass,
                double* b, const uint8_t* dirichlet, cudaStream_t s) {
    if (n == 0) return;
    k_fs_predict<<<grid_for(n, 128), 128, 0, s>>>(n, cm, el, off, inc, um, wall, P, dt, ustar, mass);
    SB_LAUNCH_CHECK();
    k_fs_rhs<<<grid_for(n, 128), 128, 0, s>>>(n, cm, el, off, inc, ustar, dirichlet, P.rho / dt, b);
    SB_LAUNCH_CHECK();
}

void fs_correct(uint32_t n, const float4* cm, const uint4* el, const uint32_t* off, const uint32_t* inc,
                const double* p, const double* mass, const double* ustar, const uint8_t* wall, const uint32_t* perm,
                const FsParams& P, double dt, float alpha, double* u_p, double* xyz_p, float4* pts4, cudaStream_t s) {
    if (n == 0) return;
    k_fs_correct<<<grid_for(n, 128), 128, 0, s>>>(n, cm, el, off, inc, p, mass, ustar, wall, perm, P, dt, dt / P.rho,
                                                  alpha, u_p, xyz_p, pts4);
    SB_LAUNCH_CHECK();
}

}  // namespace sb
