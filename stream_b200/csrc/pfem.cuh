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

}  // namespace sb
