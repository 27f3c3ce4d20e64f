// PFEM particle advection under an analytic divergence-free field.
//
// Taylor-Green field in a rotated, shifted frame x' = R (x - c):
//   u'(x') = amp (sin kx' cos ky' cos kz', -cos kx' sin ky' cos kz', 0),
//   u(x)   = R^T u'(x')
// (divergence-free for any rotation R).  Positions are FP64; explicit Euler
// steps.  The reference has no advection (it meshes given clouds).
#pragma once

#include "common.cuh"

namespace sb {

struct TaylorGreen {
    double R[9];   // row-major rotation
    double c[3];   // frame origin
    double k;      // wavenumber
    double amp;    // amplitude
};

// steps Euler steps of dt on xyz (device, n x 3 FP64, in place); when out4 is
// non-null it also receives (x, y, z, alpha) as float4 for the mesher.
void advect_taylor_green(uint32_t n, double* xyz, const TaylorGreen& f, double dt, uint32_t steps, float alpha,
                         float4* out4, cudaStream_t s);

// The pressure carried from step to step in particle order (particles keep
// their index; mesh nodes are in the mesher's Morton order, perm[m] = particle
// of node m).  to_particles: p[perm[m]] = x[m].  from_particles: the next
// step's initial guess x[m] = p[perm[m]], 0 on Dirichlet rows (is_bnd[m]).
void pressure_to_particles(uint32_t n, const uint32_t* perm, const double* x, double* p, cudaStream_t s);
void pressure_from_particles(uint32_t n, const uint32_t* perm, const double* p, const uint8_t* is_bnd, double* x,
                             cudaStream_t s);

// ---- fractional-step dynamics (pfem_fs.cu) ---------------------------------
// Incompressible flow of the particles in an axis-aligned box with gravity
// and viscosity, one projection step per remesh (Chorin's fractional step on
// the P1 mesh of the particles):
//   u*  = u + dt (g + nu lap u)                      (explicit, lumped mass)
//   K p = -(rho/dt) D u*                             (p = 0 on the free surface
//                                                     away from the walls)
//   u   = u* - (dt/rho) grad p,   x += dt u          (lumped gradient)
// Normal velocity components vanish at the walls (nodes within wall_tol of a
// box face; those keep the natural pressure condition), and a particle that
// leaves the box is put back on its face.  The reference has no such step.
struct FsParams {
    double g[3];
    double nu, rho;
    double lo[3], hi[3];
    double wall_tol;
};

// float4 (x, y, z, alpha) of FP64 particle positions, for the mesher.
void pack_particles(uint32_t n, const double* xyz, float alpha, float4* out4, cudaStream_t s);
// Mesh node m (Morton order, perm[m] = its particle): um[m] = u_p[perm[m]],
// wall bits, and the pressure Dirichlet flag (free surface, not at a wall).
void fs_gather(uint32_t n, const uint32_t* perm, const double* u_p, const float4* cm, const uint8_t* is_bnd,
               const FsParams& P, double* um, uint8_t* wall, uint8_t* dirichlet, cudaStream_t s);
// Predictor u* and lumped mass over the assembly's node-to-element incidence
// (off, inc), then the pressure load b.
void fs_predict(uint32_t n, const float4* cm, const uint4* el, const uint32_t* off, const uint32_t* inc,
                const double* um, const uint8_t* wall, const FsParams& P, double dt, double* ustar, double* mass,
                double* b, const uint8_t* dirichlet, cudaStream_t s);
// Correction, particle move and wall handling; writes velocity, position and
// the mesher's float4 in particle order.
void fs_correct(uint32_t n, const float4* cm, const uint4* el, const uint32_t* off, const uint32_t* inc,
                const double* p, const double* mass, const double* ustar, const uint8_t* wall, const uint32_t* perm,
                const FsParams& P, double dt, float alpha, double* u_p, double* xyz_p, float4* pts4, cudaStream_t s);

}  // namespace sb
