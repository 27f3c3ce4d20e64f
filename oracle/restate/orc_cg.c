// Oracle (test infrastructure only): plain-C restatement of the reference's
// FP32 conjugate gradient, src/numerics/conjugate_gradient.cpp:61-208, with the
// Jacobi preconditioner of src/numerics/preconditioner_jacobi.cpp:33-60.
// Dot products are summed pairwise (the shape of a device reduction); the
// reference's device reduction order is not specified, so FP32 results agree
// with it to rounding, not bit for bit.
#include "stream_oracle.h"

#include <math.h>
#include <stdlib.h>

static float psum(const float* v, uint32_t n) {
    if (n <= 8) { float s = 0.0f; for (uint32_t i = 0; i < n; ++i) s += v[i]; return s; }
    const uint32_t h = n / 2;
    return psum(v, h) + psum(v + h, n - h);
}
static float dot(const float* a, const float* b, float* tmp, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) tmp[i] = a[i] * b[i];
    return psum(tmp, n);
}
static void spmv(uint32_t n, const uint32_t* row, const uint32_t* col, const float* val,
                 const float* x, float* y) {
    for (uint32_t i = 0; i < n; ++i) {
        float s = 0.0f;
        for (uint32_t k = row[i]; k < row[i + 1]; ++k) s += val[k] * x[col[k]];
        y[i] = s;
    }
}

uint32_t orc_cg_f32(uint32_t n, const uint32_t* row, const uint32_t* col, const float* val,
                    const float* b, float* x, int jacobi) {
    float* r = (float*)malloc((size_t)n * 4);
    float* d = (float*)malloc((size_t)n * 4);
    float* d1 = (float*)malloc((size_t)n * 4);
    float* s = (float*)malloc((size_t)n * 4);
    float* idg = (float*)malloc((size_t)n * 4);
    float* tmp = (float*)malloc((size_t)n * 4);
    for (uint32_t i = 0; i < n; ++i) {
        idg[i] = 0.0f;
        for (uint32_t k = row[i]; k < row[i + 1]; ++k)
            if (col[k] == i) { idg[i] = 1.0f / val[k]; break; }
    }
    spmv(n, row, col, val, x, d1);
    for (uint32_t i = 0; i < n; ++i) r[i] = b[i] - d1[i];
    for (uint32_t i = 0; i < n; ++i) d[i] = jacobi ? r[i] * idg[i] : r[i];
    float sq = jacobi ? dot(r, d, tmp, n) : dot(r, r, tmp, n);
    uint32_t it = 0;
    do {
        spmv(n, row, col, val, d, d1);
        const float alpha = sq / dot(d, d1, tmp, n);
        for (uint32_t i = 0; i < n; ++i) { x[i] += alpha * d[i]; r[i] -= alpha * d1[i]; }
        const float old = sq;
        if (jacobi) {
            for (uint32_t i = 0; i < n; ++i) s[i] = r[i] * idg[i];
            sq = dot(r, s, tmp, n);
        } else {
            sq = dot(r, r, tmp, n);
        }
        const float beta = sq / old;
        for (uint32_t i = 0; i < n; ++i) d[i] = (jacobi ? s[i] : r[i]) + beta * d[i];
    } while (sqrtf(sq) > 1e-6f && it++ < 10000);
    free(r); free(d); free(d1); free(s); free(idg); free(tmp);
    return it;
}
