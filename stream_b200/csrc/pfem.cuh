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

}  // namespace sb
