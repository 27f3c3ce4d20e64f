// Particle advection for the PFEM step loop (see pfem.cuh).
#include "pfem.cuh"

namespace sb {
namespace {

__device__ __forceinline__ void tg_velocity(const TaylorGreen& f, double x, double y, double z, double& ux, double& uy,
                                            double& uz) {
    const double dx = x - f.c[0], dy = y - f.c[1], dz = z - f.c[2];
    const double xp = f.R[0] * dx + f.R[1] * dy + f.R[2] * dz;
    const double yp = f.R[3] * dx + f.R[4] * dy + f.R[5] * dz;
    const double zp = f.R[6] * dx + f.R[7] * dy + f.R[8] * dz;
    double sx, cx, sy, cy, sz, cz;
    sincos(f.k * xp, &sx, &cx);
    sincos(f.k * yp, &sy, &cy);
    sincos(f.k * zp, &sz, &cz);
    (void)sz;
    const double u0 = f.amp * sx * cy * cz, u1 = -f.amp * cx * sy * cz;
    // u = R^T u'
    ux = f.R[0] * u0 + f.R[3] * u1;
    uy = f.R[1] * u0 + f.R[4] * u1;
    uz = f.R[2] * u0 + f.R[5] * u1;
}

__global__ void __launch_bounds__(256) k_advect_tg(uint32_t n, double* __restrict__ xyz, TaylorGreen f, double dt,
                                                   uint32_t steps, float alpha, float4* __restrict__ out4) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
    for (uint32_t s = 0; s < steps; ++s) {
        double ux, uy, uz;
        tg_velocity(f, x, y, z, ux, uy, uz);
        x += dt * ux;
        y += dt * uy;
        z += dt * uz;
    }
    xyz[3 * (size_t)i] = x;
    xyz[3 * (size_t)i + 1] = y;
    xyz[3 * (size_t)i + 2] = z;
    if (out4) out4[i] = make_float4((float)x, (float)y, (float)z, alpha);
}

__global__ void k_pressure_to_particles(uint32_t n, const uint32_t* __restrict__ perm, const double* __restrict__ x,
                                        double* __restrict__ p) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n) p[perm[m]] = x[m];
}

__global__ void k_pressure_from_particles(uint32_t n, const uint32_t* __restrict__ perm, const double* __restrict__ p,
                                          const uint8_t* __restrict__ is_bnd, double* __restrict__ x) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n) x[m] = is_bnd[m] ? 0.0 : p[perm[m]];
}

}  // namespace

void pressure_to_particles(uint32_t n, const uint32_t* perm, const double* x, double* p, cudaStream_t s) {
    if (n == 0) return;
    k_pressure_to_particles<<<grid_for(n, 256), 256, 0, s>>>(n, perm, x, p);
    SB_LAUNCH_CHECK();
}

void pressure_from_particles(uint32_t n, const uint32_t* perm, const double* p, const uint8_t* is_bnd, double* x,
                             cudaStream_t s) {
    if (n == 0) return;
    k_pressure_from_particles<<<grid_for(n, 256), 256, 0, s>>>(n, perm, p, is_bnd, x);
    SB_LAUNCH_CHECK();
}

void advect_taylor_green(uint32_t n, double* xyz, const TaylorGreen& f, double dt, uint32_t steps, float alpha,
                         float4* out4, cudaStream_t s) {
    if (n == 0) return;
    k_advect_tg<<<grid_for(n, 256), 256, 0, s>>>(n, xyz, f, dt, steps, alpha, out4);
    SB_LAUNCH_CHECK();
}

}  // namespace sb
